/*
 * nise2dfft — 2DFFT-compatible driver for the B200 engine.
 *
 * Usage: nise2dfft <inputfile>   (the same keyword file the reference's 2DFFT
 * program reads, run in the directory holding the R*.dat response files)
 *
 * Writes Rw*.dat, 2D.*.dat and PP.*.dat like 2DFFT (2DFFT.c:20-830), with the
 * 2D transforms on the device chosen by NISE_DEVICE (default 0).
 */
#include <stdio.h>
#include <stdlib.h>

#include "nise_b200.h"

int main(int argc, char *argv[]) {
    if (argc != 2) {
        printf("Specify input file name on command line!\n");
        printf("Program terminated!\n");
        return 1;
    }
    const char *dev = getenv("NISE_DEVICE");
    int rc = nise_2dfft_files(argv[1], dev ? atoi(dev) : 0);
    if (rc != NISE_OK) {
        fprintf(stderr, "2D FFT failed (status %d): %s\n", rc, nise_global_error());
        return 1;
    }
    return 0;
}
