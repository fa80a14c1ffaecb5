/* Oracle build variant — TEST INFRASTRUCTURE ONLY.
 *
 * Force-included (g++ -include) when compiling the reference sources into
 * oracle/_ref/libmelon3d_ref_cr.so.  The reference calls libm's float sinf,
 * cosf and atan2f on a few rare paths (exponential-map integration of
 * spins faster than ~9.6 rad/s at 240 Hz substeps, the matching log map,
 * hinge angles).  glibc's float versions are not correctly rounded, so no
 * other implementation can reproduce their last bit.  This variant evaluates
 * them in double precision and rounds once, exactly as the GPU kernels do,
 * so that a bit-level comparison with it isolates every other source of
 * difference.  The stock oracle (libmelon3d_ref.so) keeps glibc's versions
 * and is compared with a tolerance on those paths.
 */
#ifndef M3D_ORACLE_CR_LIBM_H
#define M3D_ORACLE_CR_LIBM_H
#include <math.h>
#ifdef __cplusplus
#include <cmath>
#endif
static inline float m3d_oracle_sinf(float x) { return (float)sin((double)x); }
static inline float m3d_oracle_cosf(float x) { return (float)cos((double)x); }
static inline float m3d_oracle_atan2f(float y, float x) { return (float)atan2((double)y, (double)x); }
#define sinf m3d_oracle_sinf
#define cosf m3d_oracle_cosf
#define atan2f m3d_oracle_atan2f
#endif
