/*
 * ref_rysdump.c -- test infrastructure: prints the reference's own Rys
 * roots (as t^2 = u/(1+u), rys.c:317-321 stores u) and weights for the root
 * count given on the command line, one line per T read from stdin, by
 * calling Rys_findRoots (rys.c:2217-2244) from the reference's rys.o.
 */
#include <stdio.h>
#include <stdlib.h>
#include "rys.h"

int main(int argc, char **argv)
{
    int n = argc > 1 ? atoi(argv[1]) : 1, i;
    double T;
    while (scanf("%lf", &T) == 1) {
        const double *r, *w;
        Rys_findRoots(n, T);
        r = RysRoots();
        w = RysWeights();
        for (i = 0; i < n; i++) printf("%.17g %.17g ", r[i] / (1.0 + r[i]), w[i]);
        printf("\n");
    }
    return 0;
}
