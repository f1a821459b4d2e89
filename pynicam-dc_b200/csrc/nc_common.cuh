// Device data model of the NICAM-DC dynamics step on one B200.
//
// Regional fields: one array per variable, layout [l][k][j][i] with i
// fastest (the Fortran/fio (gall, kall, lall) order, ij = j*gall_1d + i), so a
// warp of threads on consecutive i issues coalesced 128-byte loads and the
// 7-point hexagonal stencil touches rows j-1, j, j+1 of the same k-plane.
// Horizontal (k-independent) coefficients: [c][l][j][i].  Pole fields keep the
// reference's (g, k, l) C-order (g = 0 pole point, 1..5 its neighbours).
//
// Every kernel is a "column" kernel: one thread owns one (i, j, l) column and
// walks k, so k-independent coefficients are loaded once into registers and
// the vertical recurrences (Thomas solve, limiter) stay in registers.
//
// Two forms of every kernel, selected per handle: float64 (R = double) and
// the mixed form (R = float: float32 fields, metrics and arithmetic, with the
// Thomas elimination, the pressure / density deviations and the mass sums in
// float64).  The float64 arithmetic follows the numpy reference op-for-op
// (same association order, no FMA contraction: the library is built
// -fmad=false), which is what makes the float64 step bit-identical to the
// reference.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define NC_MAXK 128
#define NC_MAXNQ 32
#define NC_MAXQW 6   // water tracers (RAIN_TYPE COLD: vapour, cloud, rain, ice, snow, graupel)

namespace nc {

struct Dims {
  int G;      // gall_1d (region tile edge incl. 1-cell halo)
  int KA;     // kall
  int L;      // regions on this device
  int LP;     // pole regions (2)
  int kmin, kmax, gmin, gmax;
  int nq;
  long long plane;   // G*G
  long long npt;     // L*KA*G*G
  long long npt2;    // L*G*G
  int npl;           // 6*KA*LP
  // the same sizes as 32-bit ints: device index arithmetic is 32-bit (the
  // host rejects grids where 6*npt would not fit)
  int planei, npti, npt2i;
};

// Physical / run constants (identical names to the reference's CONST_*).
// R is the arithmetic type of the kernels that read them: the float64 form
// uses ConstsT<double> (cC) throughout; the mixed form loads a float copy
// (cCf) for its float32 kernels and keeps cC for its float64 parts.
template <class R>
struct ConstsT {
  R GRAV, Rdry, CVdry, CPdry, Rvap, OHM, EPS, HUGE_, rscale, alpha;
  R Kh, divdamp_coef, hdiff_fact_rho, CVW0, PRE00;
  R CVW[NC_MAXQW];   // specific heats of the water tracers 0..nqw-1
  int nqw;           // water tracers (NQW_END + 1; NQW_STR = I_QV = 0)
  int gam_unit;   // RGAM, RGAMH and GAM2H are 1 everywhere (shallow atmosphere)
  // rounded reciprocals and their tails, RN(1/b) and RN(1/b - RN(1/b)), of the
  // divisors rscale and 3 (see div_by)
  R rsc_h, rsc_l, third_h, third_l;
  R afact[NC_MAXK], bfact[NC_MAXK], cfact[NC_MAXK], dfact[NC_MAXK];
  R rdgz[NC_MAXK], rdgzh[NC_MAXK];
  // hyperdiffusion NONLINEAR1 (hdiff_nl): Kh = clip(nl_c1 |lapT| / 300 nl_area,
  // nl_min, nl_khmax[k]), nl_c1 = 2 AREA_ave^2 / dtl
  int hdiff_nl;
  R nl_c1, nl_area, nl_min;
  R nl_khmax[NC_MAXK];
  // Rayleigh sponge (rayleigh): coefficients on full and half levels
  int rayleigh, rayleigh_only_w;
  R ray_c[NC_MAXK], ray_ch[NC_MAXK];
};
using Consts = ConstsT<double>;

// Geometry on the device.  Regional 3-D metrics [l][k][j][i]; 2-D coefficient
// planes [c][l][j][i].  Pole arrays in reference layout.  GeomT<double> (cG)
// holds the float64 arrays; the mixed form stores a float32 copy of every
// array (GeomT<float>, cGf) and its kernels read that one.
template <class R>
struct GeomT {
  // 3-D vertical metrics
  const R *GSGAM2, *GSGAM2H, *RGSGAM2, *RGSGAM2H, *RGSQRTH, *RGAM, *RGAMH, *GAM2H, *PHI;
  const R *C2W;     // 2 comps
  const R *W2C;     // 2 comps
  const R *C2WGz;   // 6 comps
  const R *rho_bs, *pre_bs, *tem_bs;
  // 2-D horizontal coefficients
  const R *coef_div;   // 21 planes (d*7+m)
  const R *coef_grad;  // 21 planes
  const R *coef_lap;   // 7
  const R *coef_intp;  // 18 planes ((d*3+p)*2+t)
  const R *intp_w;     // 18 planes ((d*3+m)*2+t): the diffusion's vertex weights formed from coef_intp
  const R *coef_diff;  // 18 planes (d*6+m)
  const R *GRD_x;      // 3
  const R *GRD_xr;     // 9 (face*3+d)
  const R *GMTR_t;     // 6 (t*3 + (W-2))
  const R *GMTR_a;     // 9 (face*3 + HN)
  const R *GMTR_p;     // 1 (P_RAREA)
  const int *pntmask;  // [l][2]
  const int *have_sgp; // [l]
  // pole (reference layouts)
  const R *GSGAM2_pl, *GSGAM2H_pl, *RGSGAM2_pl, *RGSGAM2H_pl, *RGSQRTH_pl, *RGAM_pl, *RGAMH_pl,
      *GAM2H_pl, *PHI_pl;
  const R *C2W_pl, *W2C_pl, *C2WGz_pl;   // (g,k,l,c)
  const R *rho_bs_pl, *pre_bs_pl, *tem_bs_pl;
  const R *coef_div_pl;   // (g,l,3)
  const R *coef_grad_pl;  // (g,l,3)
  const R *coef_lap_pl;   // (g,l)
  const R *coef_intp_pl;  // (g,l,3,3)
  const R *coef_diff_pl;  // (g,l,3)
  const R *GRD_x_pl;      // (g,l,3)
  const R *GRD_xr_pl;     // (g,l,3)
  const R *GMTR_t_pl;     // (g,l,5)
  const R *GMTR_a_pl;     // (g,l,18)
  const R *GMTR_p_pl;     // (g,l,8)
};
using Geom = GeomT<double>;

// The library is one translation unit (nc_api.cu includes every kernel
// header), so the constant-memory symbols are defined here.
__constant__ Dims cD;
__constant__ Consts cC;
__constant__ Geom cG;
__constant__ ConstsT<float> cCf;
__constant__ GeomT<float> cGf;

// a non-deduced context: a parameter of type Id<R>::type converts to R
// instead of taking part in deducing R
template <class T>
struct Id {
  using type = T;
};

// constants and geometry of arithmetic / storage type R
template <class R> __device__ __forceinline__ const ConstsT<R>& consts();
template <> __device__ __forceinline__ const ConstsT<double>& consts<double>() { return cC; }
template <> __device__ __forceinline__ const ConstsT<float>& consts<float>() { return cCf; }
template <class R> __device__ __forceinline__ const GeomT<R>& geom();
template <> __device__ __forceinline__ const GeomT<double>& geom<double>() { return cG; }
template <> __device__ __forceinline__ const GeomT<float>& geom<float>() { return cGf; }
// inside a kernel templated on R
#define CC (consts<R>())
#define CG (geom<R>())

// Resident-block targets of the launch bounds: the float64 instances keep the
// values measured for them; the float32 instances need about half the
// registers and take their own targets, from a sweep of 4-16 blocks per SM
// at gl08 on B200 (per-kernel event times; the ones left at the float64
// value were slower at every higher target).
#define NC_MINB(R, f64, f32) (sizeof(R) == 8 ? (f64) : (f32))
#ifndef NC_F32_DIAG
#define NC_F32_DIAG 9
#endif
#ifndef NC_F32_ADVMOM
#define NC_F32_ADVMOM 4
#endif
#ifndef NC_F32_HDIFF2
#define NC_F32_HDIFF2 4
#endif
#ifndef NC_F32_VP0H
#define NC_F32_VP0H 5
#endif
#ifndef NC_F32_VP0C
#define NC_F32_VP0C 4
#endif
#ifndef NC_F32_PATH1
#define NC_F32_PATH1 6
#endif
#ifndef NC_F32_VIMAINA
#define NC_F32_VIMAINA 6
#endif
#ifndef NC_F32_VISOLVE
#define NC_F32_VISOLVE 9
#endif
#ifndef NC_F32_VIENERGY
#define NC_F32_VIENERGY 12
#endif

// The gamma factors of the vertical metrics: RGAM, RGAMH, GAM2H (regional or
// pole) at index p.  With a shallow atmosphere every value is exactly 1 (the
// host checks each element at set-up and sets gam_unit); the factor is then
// not loaded, and x * 1.0 == x leaves every product bit-for-bit unchanged.
template <class R>
__device__ __forceinline__ R gam_at(const R* a, int p) { return cC.gam_unit ? R(1) : a[p]; }
template <class R>
__device__ __forceinline__ R gam_at_ldg(const R* a, int p) { return cC.gam_unit ? R(1) : __ldg(a + p); }

// x / b for a divisor fixed before the launch, with the same bits as the IEEE
// division x / b for finite x whose quotient is in the normal range.  From
// bh = RN(1/b) and bl = RN(1/b - bh), q0 = RN(x*bh + x*bl) is within one ulp
// of x/b (the double-word reciprocal of Brisebarre, Muller and Raina,
// "Accelerating correctly rounded floating-point division when the divisor is
// known in advance", IEEE Trans. Computers 53(8), 2004); the remainder
// x - b*q0 is then exact, and one correction RN(q0 + r*bh) gives the correctly
// rounded quotient (Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990).  A zero x takes
// its quotient's sign from x*bh.  Three FMAs and a multiply instead of a
// general division.
__device__ __forceinline__ double div_by(double x, double b, double bh, double bl) {
  const double q0 = __fma_rn(x, bh, __dmul_rn(x, bl));
  const double r = __fma_rn(-q0, b, x);
  const double q = __fma_rn(r, bh, q0);
  return (x == 0.0) ? __dmul_rn(x, bh) : q;
}
// x / rscale and x / 3.0
__device__ __forceinline__ double div_r(double x) { return div_by(x, cC.rscale, cC.rsc_h, cC.rsc_l); }
__device__ __forceinline__ double div3(double x) { return div_by(x, 3.0, cC.third_h, cC.third_l); }

// The same division for a divisor computed at run time that several quotients
// share: bh = RN(1/b) from the correctly rounded reciprocal __drcp_rn, and the
// tail RN((1 - b*bh) * bh) (1 - b*bh is exact), which is within a relative
// 2^-52 of 1/b - bh, so RN(x*bh + x*bl) is still within one ulp of x/b and the
// correction step rounds the quotient correctly.
struct Recip {
  double b, h, l;
};
__device__ __forceinline__ Recip recip_of(double b) {
  Recip r;
  r.b = b;
  r.h = __drcp_rn(b);
  r.l = __dmul_rn(__fma_rn(-r.h, b, 1.0), r.h);
  return r;
}
__device__ __forceinline__ double div_by(double x, const Recip& r) { return div_by(x, r.b, r.h, r.l); }

// The float32 forms used by the mixed-precision kernels: a multiplication by
// the rounded reciprocal (within 1.5 ulp of the quotient; the float32 kernels
// are not bit-for-bit with anything, so the correction step is left out).
__device__ __forceinline__ float div_r(float x) { return x * cCf.rsc_h; }
__device__ __forceinline__ float div3(float x) { return x * cCf.third_h; }
struct RecipF {
  float h;
};
__device__ __forceinline__ RecipF recip_of(float b) { return RecipF{__frcp_rn(b)}; }
__device__ __forceinline__ float div_by(float x, const RecipF& r) { return x * r.h; }

// ---- indexing -------------------------------------------------------------
__device__ __forceinline__ int ix(int i, int j, int k, int l) {
  return ((l * cD.KA + k) * cD.G + j) * cD.G + i;
}
// plane c of a 2-D coefficient array: c * (L*G*G) + cell offset, written so
// that the cell offset is shared between the planes of one cell
__device__ __forceinline__ int ix2(int c, int i, int j, int l) {
  return c * cD.npt2i + ((l * cD.G + j) * cD.G + i);
}
// pole (g, k, l)
__device__ __forceinline__ int ipl(int g, int k, int lp) { return (g * cD.KA + k) * cD.LP + lp; }
template <class R>
__device__ __forceinline__ R P2(const R* a, int c, int i, int j, int l) { return a[ix2(c, i, j, l)]; }
// the same through the read-only (non-coherent) path: the planes are constant
// after set-up, and the compiler may batch these loads ahead of shared-memory
// stores.  Used where that measured faster (path 1, 3-D divergence damping,
// tracer horizontal flux); where it raised register pressure into spills
// (momentum advection, vp0 horizontal terms) the plain load is kept.
template <class R>
__device__ __forceinline__ R P2c(const R* a, int c, int i, int j, int l) { return __ldg(a + ix2(c, i, j, l)); }

// 7-point neighbour offsets in the reference's coefficient order:
// (i,j) (i+1,j) (i+1,j+1) (i,j+1) (i-1,j) (i-1,j-1) (i,j-1)
__device__ __constant__ static const int kNbI[7] = {0, 1, 1, 0, -1, -1, 0};
__device__ __constant__ static const int kNbJ[7] = {0, 0, 1, 1, 0, -1, -1};

__device__ __forceinline__ bool interior(int i, int j) {
  return i >= 1 && i <= cD.G - 2 && j >= 1 && j <= cD.G - 2;
}

// qd and cv from the water mixing ratios q0 = q(0), q(1) .. q(nqw-1)
// (kernels/diag.py:97-115: both sums in index order; with one water tracer
// qd = 1 - q0 and cv = q0 CVW0 + qd CVdry)
template <class F>
__device__ __forceinline__ void moist_qd_cv(F q, double q0, double& qd, double& cv) {
  double sq = q0, sc = q0 * (double)cC.CVW[0];
  for (int n = 1; n < cC.nqw; ++n) {
    const double x = q(n);
    sq = sq + x;
    sc = sc + x * (double)cC.CVW[n];
  }
  qd = 1.0 - sq;
  cv = sc + qd * cC.CVdry;
}

// Column thread mapping: thread -> (i, j, l).  Returns false for surplus threads.
__device__ __forceinline__ bool col_of(int t, int& i, int& j, int& l) {
  if (t >= cD.npt2i) return false;
  i = t % cD.G;
  int r = t / cD.G;
  j = (int)(r % cD.G);
  l = (int)(r / cD.G);
  return true;
}

}  // namespace nc
