// Point/column building blocks shared by the dynamics kernels.  Each function
// restates one reference expression with the reference's association order
// (pynicamdc/nhm/dynamics/kernels/*.py); comments cite the file:line.
#pragma once
#include "nc_common.cuh"

namespace nc {

// numpy elementwise minimum/maximum: on ties the second operand is returned
template <class R> __device__ __forceinline__ R npmin(R a, R b) { return (a < b) ? a : b; }
template <class R> __device__ __forceinline__ R npmax(R a, R b) { return (a > b) ? a : b; }
// Python builtin min/max: on ties the first operand is kept
template <class R> __device__ __forceinline__ R pymin(R a, R b) { return (b < a) ? b : a; }
template <class R> __device__ __forceinline__ R pymax(R a, R b) { return (b > a) ? b : a; }

// Column accessor: value index = base + k*ks.  Regional columns use
// base = ix(i,j,0,l), ks = G*G; pole columns base = g*KA*LP + lp, ks = LP.
// Multi-component metrics: regional comp c lives at c*npt + idx, pole comps are
// interleaved (idx*nc + c).
struct Col {
  int base, ks;
  bool pole;
  __device__ __forceinline__ int at(int k) const { return base + k * ks; }
};

__device__ __forceinline__ Col col_reg(int i, int j, int l) {
  Col c;
  c.base = ix(i, j, 0, l);
  c.ks = cD.planei;
  c.pole = false;
  return c;
}
__device__ __forceinline__ Col col_pl(int g, int lp) {
  Col c;
  c.base = g * cD.KA * cD.LP + lp;
  c.ks = cD.LP;
  c.pole = true;
  return c;
}

// Thread -> column for a launch over regional columns (pole == 0) or over the
// 6*LP pole columns (pole != 0).  The caller passes pointers of the matching kind.
__device__ __forceinline__ bool map_col(int pole, int t, int& i, int& j, int& l, int& g, int& lp) {
  if (!pole) {
    g = lp = 0;
    return col_of(t, i, j, l);
  }
  if (t >= 6 * cD.LP) return false;
  g = (int)(t / cD.LP);
  lp = (int)(t % cD.LP);
  i = j = l = 0;
  return true;
}

// Metric selection by column kind
template <class R>
struct MetT {
  const R *GSGAM2, *GSGAM2H, *RGSGAM2, *RGSGAM2H, *RGSQRTH, *RGAM, *RGAMH, *GAM2H, *PHI;
  const R *C2W, *W2C, *C2WGz, *rho_bs, *pre_bs, *tem_bs;
};
template <class R>
__device__ __forceinline__ MetT<R> met_of(bool pole) {
  const GeomT<R>& cG = geom<R>();
  MetT<R> m;
  if (!pole) {
    m.GSGAM2 = cG.GSGAM2; m.GSGAM2H = cG.GSGAM2H; m.RGSGAM2 = cG.RGSGAM2; m.RGSGAM2H = cG.RGSGAM2H;
    m.RGSQRTH = cG.RGSQRTH; m.RGAM = cG.RGAM; m.RGAMH = cG.RGAMH; m.GAM2H = cG.GAM2H; m.PHI = cG.PHI;
    m.C2W = cG.C2W; m.W2C = cG.W2C; m.C2WGz = cG.C2WGz;
    m.rho_bs = cG.rho_bs; m.pre_bs = cG.pre_bs; m.tem_bs = cG.tem_bs;
  } else {
    m.GSGAM2 = cG.GSGAM2_pl; m.GSGAM2H = cG.GSGAM2H_pl; m.RGSGAM2 = cG.RGSGAM2_pl;
    m.RGSGAM2H = cG.RGSGAM2H_pl; m.RGSQRTH = cG.RGSQRTH_pl; m.RGAM = cG.RGAM_pl; m.RGAMH = cG.RGAMH_pl;
    m.GAM2H = cG.GAM2H_pl; m.PHI = cG.PHI_pl; m.C2W = cG.C2W_pl; m.W2C = cG.W2C_pl; m.C2WGz = cG.C2WGz_pl;
    m.rho_bs = cG.rho_bs_pl; m.pre_bs = cG.pre_bs_pl; m.tem_bs = cG.tem_bs_pl;
  }
  return m;
}
// component c (of nc) of a multi-component metric at column level k
template <class R>
__device__ __forceinline__ R mc(const R* a, const Col& c, int comp, int ncomp, int k) {
  return c.pole ? a[c.at(k) * ncomp + comp] : a[comp * cD.npti + c.at(k)];
}

// ---- horizontal 7-point operators (regional, interior (i,j) only) ---------

// divergence of (vx,vy,vz) at (i,j,k,l) given a functor returning the three
// components at a neighbour: kernels/fluxconv.py:52-78
template <class R, class F>
__device__ __forceinline__ R div7(int i, int j, int k, int l, F vel) {
  R acc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    R s = R(0);
#pragma unroll
    for (int m = 0; m < 7; ++m) {
      R v = vel(i + kNbI[m], j + kNbJ[m], k, d);
      R t = P2(CG.coef_div, d * 7 + m, i, j, l) * v;
      s = (m == 0) ? t : s + t;
    }
    acc[d] = s;
  }
  return acc[0] + acc[1] + acc[2];
}

// gradient components (kernels/oprtgradient.py:45-70): np.sum over the 7
// stencil points, left to right
template <class R, class F>
__device__ __forceinline__ void grad7(int i, int j, int k, int l, F scl, R out[3]) {
  R s[7];
#pragma unroll
  for (int m = 0; m < 7; ++m) s[m] = scl(i + kNbI[m], j + kNbJ[m], k);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    R a = P2(CG.coef_grad, d * 7 + 0, i, j, l) * s[0];
#pragma unroll
    for (int m = 1; m < 7; ++m) a = a + P2(CG.coef_grad, d * 7 + m, i, j, l) * s[m];
    out[d] = a;
  }
}

// laplacian (kernels/oprtlaplacian.py:41-55)
template <class R, class F>
__device__ __forceinline__ R lap7(int i, int j, int k, int l, F scl) {
  R a = P2(CG.coef_lap, 0, i, j, l) * scl(i, j, k);
#pragma unroll
  for (int m = 1; m < 7; ++m) a = a + P2(CG.coef_lap, m, i, j, l) * scl(i + kNbI[m], j + kNbJ[m], k);
  return a;
}

// tangent-plane projection of one vector at an interior point
// (kernels/horizontalizevec.py:51-54)
template <class R>
__device__ __forceinline__ void horiz_reg(int i, int j, int l, R& vx, R& vy, R& vz) {
  R gx = P2(CG.GRD_x, 0, i, j, l), gy = P2(CG.GRD_x, 1, i, j, l), gz = P2(CG.GRD_x, 2, i, j, l);
  R prd = div_r(vx * gx + vy * gy + vz * gz);
  R nx = vx - div_r(prd * gx);
  R ny = vy - div_r(prd * gy);
  R nz = vz - div_r(prd * gz);
  vx = nx; vy = ny; vz = nz;
}
// pole projection (kernels/horizontalizevec.py:67-71)
template <class R>
__device__ __forceinline__ void horiz_pl(int g, int lp, R& vx, R& vy, R& vz) {
  const R* X = CG.GRD_x_pl;
  R gx = X[(g * cD.LP + lp) * 3 + 0], gy = X[(g * cD.LP + lp) * 3 + 1], gz = X[(g * cD.LP + lp) * 3 + 2];
  R prd = div_r(vx * gx) + div_r(vy * gy) + div_r(vz * gz);
  R nx = vx - div_r(prd * gx);
  R ny = vy - div_r(prd * gy);
  R nz = vz - div_r(prd * gz);
  vx = nx; vy = ny; vz = nz;
}

// ---- vertical pieces ------------------------------------------------------

// horizontal part of the half-level mass flux (kernels/fluxconv.py:142-151):
// (sum of C2WfactGz * fluxes at k, k-1) * RGAMH(k)
template <class R, class F>
__device__ __forceinline__ R vmh_horiz(const Col& c, const MetT<R>& m, int k, F flux) {
  R h = mc(m.C2WGz, c, 0, 6, k) * flux(k, 0) + mc(m.C2WGz, c, 1, 6, k) * flux(k - 1, 0) +
             mc(m.C2WGz, c, 2, 6, k) * flux(k, 1) + mc(m.C2WGz, c, 3, 6, k) * flux(k - 1, 1) +
             mc(m.C2WGz, c, 4, 6, k) * flux(k, 2) + mc(m.C2WGz, c, 5, 6, k) * flux(k - 1, 2);
  return h * gam_at(m.RGAMH, c.at(k));
}

// total kinetic energy rhogkin at level k of one column (kernels/rhogkin.py:38-79)
template <class R, class F>
__device__ __forceinline__ R rhogkin_at(const Col& c, const MetT<R>& m, int k, F st) {
  // st(k, comp): comp 0 rhog, 1..3 rhogv{x,y,z}, 4 rhogw
  const int kmin = cD.kmin, kmax = cD.kmax;
  if (k < kmin || k > kmax) return R(0);
  R rg = st(k, 0), vx = st(k, 1), vy = st(k, 2), vz = st(k, 3);
  R kh = R(0.5) * (vx * vx + vy * vy + vz * vz) / rg;
  auto vint = [&](int kk) -> R {  // defined for kk in kmin+1..kmax, zero at kmin and kmax+1
    if (kk <= kmin || kk > kmax) return R(0);
    R den = mc(m.C2W, c, 0, 2, kk) * st(kk, 0) + mc(m.C2W, c, 1, 2, kk) * st(kk - 1, 0);
    R w = st(kk, 4);
    return R(0.5) * (w * w) / den;
  };
  return kh + mc(m.W2C, c, 0, 2, k) * vint(k + 1) + mc(m.W2C, c, 1, 2, k) * vint(k);
}

}  // namespace nc
