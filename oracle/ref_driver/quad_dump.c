/*
 * Test-infrastructure helper: prints the reference's 3D quadrature rules
 * (phgQuadGetQuad3D, src/quad.c:2914) for orders 0..6 as C99 hex floats, so
 * the restated rule tables can be compared bit-for-bit against them.
 */
#include "phg.h"
#include <stdio.h>

int
main(int argc, char *argv[])
{
    int order, i, k;

    phgInit(&argc, &argv);
    for (order = 0; order <= 6; order++) {
	QUAD *q = phgQuadGetQuad3D(order);
	printf("order %d npoints %d name %s\n", order, q->npoints, q->name);
	for (i = 0; i < q->npoints; i++) {
	    for (k = 0; k < 4; k++)
		printf("%a ", (double)q->points[4 * i + k]);
	    printf("%a\n", (double)q->weights[i]);
	}
    }
    phgFinalize();
    return 0;
}
