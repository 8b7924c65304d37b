/* CPU restatement of the reference's affine-tet acoustic WADG stage.
 *
 * ORACLE - TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or
 * calls this library; only tests/, the smoke check and bench.py's CPU
 * baseline leg use it, and only as the checker.
 *
 * The functions restate cpp/okl/WaveKernels.okl (rk_volume, rk_surface,
 * rk_update, rk_volume_bern, rk_surface_bern) and
 * cpp/okl/WaveKernelsWADG.okl (rk_update_WADG) in the reference's loop and
 * summation order.  The _f32 family reproduces the reference's FP32
 * arithmetic; the _f64 family is the same method in double precision, the
 * accuracy oracle for error-vs-FP64 figures.  Parity of this restatement is
 * pinned against the reference's own kernels (tests/golden, produced by
 * oracle/_ref from the reference sources).  Built with -ffp-contract=off so
 * the result does not depend on the host's FMA support.
 */
#define MAXNP 220   /* N <= 9 */
#define MAXNFP 55
#define MAXNQ 1000  /* Stroud rule of degree 2N+1 at N = 9 */

#define REAL float
#define SFX _f32
#include "wadg_oracle_body.h"
#undef REAL
#undef SFX

#define REAL double
#define SFX _f64
#include "wadg_oracle_body.h"
#undef REAL
#undef SFX

int ora_maxnp(void) { return MAXNP; }
int ora_maxnq(void) { return MAXNQ; }
