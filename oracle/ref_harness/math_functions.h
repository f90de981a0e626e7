/* Empty stand-in for the CUDA header of the same name that readyc.cpp
 * includes; the CPU build takes its math functions from <cmath>.  TEST
 * INFRASTRUCTURE ONLY (builds oracle/_ref). */
