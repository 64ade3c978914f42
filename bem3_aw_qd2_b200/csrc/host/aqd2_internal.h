/* Internal helpers of the host library (not part of the public API). */
#ifndef AQD2_INTERNAL_H
#define AQD2_INTERNAL_H
#include "../../../include/bem3_aw_qd2.h"
#include "../../../include/bemgpu.h"

void *aqd2_calloc(size_t n, size_t sz, const char *what);
void aqd2_malloc_node(BOUD *bd);
void aqd2_malloc_elem(BOUD *bd);
void aqd2_malloc_sub_domain(AQD2 *qd);
void aqd2_init_elem_const(BOUD *bd);
void aqd2_gauss_legendre(double *x, double *w, int n);
int aqd2_elem_plane(BOUD *bd, int e);
void aqd2_release_device(AQD2 *qd);
double aqd2_now(void);
/* point of element e (absolute id) at parameters (zeta, eta) (r_bd, d3qd2_elem.c:18) */
void aqd2_r_bd(double *r, int e, double zeta, double eta, BOUD *bd);

/* near-boundary cut-off of |grad F| in the field evaluation (CBD_CDF, d3qd2_const.h:82) */
#define AQD2_CBD_CDF 10.0

#endif
