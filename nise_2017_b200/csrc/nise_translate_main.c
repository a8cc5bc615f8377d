/*
 * nise_translate — trajectory format translation, the reference's
 * `translate` program (translate.c:25-65) on this library.
 *
 * Usage: nise_translate <inputfile>   (the reference's translate keywords)
 */
#include <stdio.h>

#include "nise_b200.h"

int main(int argc, char *argv[]) {
    if (argc < 2) {
        printf("Specify input file name on command line!\n");
        printf("Program terminated!\n");
        return 255;
    }
    printf("Using input file '%s'.\n", argv[1]);
    int rc = nise_translate(argv[1]);
    if (rc != NISE_OK) {
        fprintf(stderr, "translation failed (status %d): %s\n", rc, nise_global_error());
        return 1;
    }
    return 0;
}
