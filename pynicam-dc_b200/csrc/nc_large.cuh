// Large-step kernels of one RK stage: diagnostics + boundary conditions,
// momentum advection, hyperdiffusion and the large-step tendency.
#pragma once
#include "nc_ops.cuh"

namespace nc {

// Field bundles (device pointers, one array per variable)
template <class R>
struct Prog { R* v[6]; };   // RHOG, RHOGVX, RHOGVY, RHOGVZ, RHOGW, RHOGE

// ---------------------------------------------------------------------------
// Pre_Post: diagnostics (kernels/diag.py:53-143), BNDCND_all
// (share/mod_bndcnd.py:182-264 with kernels/bndcnd.py), th/eth and the
// deviations (mod_dynamics.py:1043-1057), then the merged velocity of the
// momentum advection (kernels/advconvmom.py:54-78).  One thread per column,
// regional and pole columns alike.
// ---------------------------------------------------------------------------
template <class R>
struct DiagArgs {
  Prog<R> P;            // in/out (ghost rows written)
  const R* Pqw[NC_MAXQW];   // the water tracers (0: vapour)
  R *pre, *tem, *vx, *vy, *vz, *w, *rho, *ein, *eth;
  double *pregd, *rhogd;   // float64 in both forms
  R *vvx, *vvy, *vvz;
};

template <class R>
__device__ void diag_column(const Col c, const MetT<R> m, const DiagArgs<R>& a, double gx, double gy, double gz) {
  const int KA = cD.KA, kmin = cD.kmin, kmax = cD.kmax;
  R** P = const_cast<R**>(a.P.v);
  for (int k = 0; k < KA; ++k) {
    int p = c.at(k);
    double RHOG = P[0][p];
    double rho = RHOG / m.GSGAM2[p];
    a.vx[p] = P[1][p] / RHOG;
    a.vy[p] = P[2][p] / RHOG;
    a.vz[p] = P[3][p] / RHOG;
    double ein = P[5][p] / RHOG;
    double q0 = a.Pqw[0][p] / RHOG;
    double qd, cv;
    moist_qd_cv([&](int n) { return (double)a.Pqw[n][p] / RHOG; }, q0, qd, cv);
    double tem = ein / cv;
    a.tem[p] = tem;
    a.pre[p] = rho * tem * (qd * cC.Rdry + q0 * cC.Rvap);
    a.rho[p] = rho;
    a.ein[p] = ein;
    if (k >= kmin + 1 && k <= kmax) {
      int pm = c.at(k - 1);
      a.w[p] = P[4][p] / (mc(m.C2W, c, 0, 2, k) * RHOG + mc(m.C2W, c, 1, 2, k) * P[0][pm]);
    }
  }
  // ---- boundary conditions: TEM top/bottom, FREE top, RIGID bottom
  const int pT = c.at(kmax + 1), pK = c.at(kmax), pKm = c.at(kmax - 1);
  const int pB = c.at(kmin - 1), pN = c.at(kmin), pNp = c.at(kmin + 1);
  double tem_top = a.tem[pK];
  double tem_btm = a.tem[pN];
  double pre_top = a.pre[pKm] - a.rho[pK] * (m.PHI[pT] - m.PHI[pKm]);
  double pre_btm = a.pre[pNp] - a.rho[pN] * (m.PHI[pB] - m.PHI[pNp]);
  double rho_top = pre_top / (cC.Rdry * tem_top);
  double rho_btm = pre_btm / (cC.Rdry * tem_btm);
  a.tem[pT] = tem_top; a.tem[pB] = tem_btm;
  a.pre[pT] = pre_top; a.pre[pB] = pre_btm;
  a.rho[pT] = rho_top; a.rho[pB] = rho_btm;
  double rgT = rho_top * m.GSGAM2[pT];
  double rgB = rho_btm * m.GSGAM2[pB];
  P[0][pT] = rgT; P[0][pB] = rgB;
  double einT = cC.CVdry * tem_top, einB = cC.CVdry * tem_btm;
  a.ein[pT] = einT; a.ein[pB] = einB;
  P[5][pT] = rgT * einT; P[5][pB] = rgB * einB;
  double rgK = P[0][pK], rgN = P[0][pN];
  double vT[3], vB[3];
  for (int d = 0; d < 3; ++d) {
    vT[d] = 1.0 * (P[1 + d][pK] / rgK) * rgT;
    vB[d] = -1.0 * (P[1 + d][pN] / rgN) * rgB;
    P[1 + d][pT] = vT[d];
    P[1 + d][pB] = vB[d];
  }
  R* dv[3] = {a.vx, a.vy, a.vz};
  for (int d = 0; d < 3; ++d) {
    dv[d][pT] = P[1 + d][pT] / P[0][pT];
    dv[d][pB] = P[1 + d][pB] / P[0][pB];
  }
  const int kT = kmax + 1;
  double rwT = -(mc(m.C2WGz, c, 0, 6, kT) * vT[0] + mc(m.C2WGz, c, 1, 6, kT) * P[1][pK] +
                 mc(m.C2WGz, c, 2, 6, kT) * vT[1] + mc(m.C2WGz, c, 3, 6, kT) * P[2][pK] +
                 mc(m.C2WGz, c, 4, 6, kT) * vT[2] + mc(m.C2WGz, c, 5, 6, kT) * P[3][pK]);
  P[4][pT] = rwT;
  P[4][pN] = 0.0;
  P[4][pB] = 0.0;
  a.w[pT] = rwT / (mc(m.C2W, c, 0, 2, kT) * rgT + mc(m.C2W, c, 1, 2, kT) * rgK);
  a.w[pN] = P[4][pN] / (mc(m.C2W, c, 0, 2, kmin) * rgN + mc(m.C2W, c, 1, 2, kmin) * rgB);
  a.w[pB] = 0.0;
  // ---- eth, deviations, merged velocity
  for (int k = 0; k < KA; ++k) {
    int p = c.at(k);
    double pre = a.pre[p], rho = a.rho[p];
    a.eth[p] = a.ein[p] + pre / rho;
    a.pregd[p] = (pre - m.pre_bs[p]) * m.GSGAM2[p];
    a.rhogd[p] = (rho - m.rho_bs[p]) * m.GSGAM2[p];
    if (k >= kmin && k <= kmax) {
      double wc = cC.cfact[k] * a.w[c.at(k + 1)] + cC.dfact[k] * a.w[p];
      a.vvx[p] = a.vx[p] + div_r(wc * gx);
      a.vvy[p] = a.vy[p] + div_r(wc * gy);
      a.vvz[p] = a.vz[p] + div_r(wc * gz);
    } else {
      a.vvx[p] = 0.0; a.vvy[p] = 0.0; a.vvz[p] = 0.0;
    }
  }
}

// diag_column with the second pass (eth, deviations, merged velocity) fused
// into the first for the levels kmin+1..kmax-1, whose inputs do not depend on
// the boundary rows: level k-1 is finished while level k is diagnosed, from
// values carried in registers.  The four levels next to and on the boundary
// rows are finished after the boundary conditions, as in diag_column.  Same
// expressions, same results.
template <class R>
__device__ void diag_column_fused(const Col c, const MetT<R> m, const DiagArgs<R>& a, double gx, double gy, double gz) {
  const int KA = cD.KA, kmin = cD.kmin, kmax = cD.kmax;
  R** P = const_cast<R**>(a.P.v);
  auto finish = [&](int k, int p, double pre, double rho, double ein, double vxk, double vyk, double vzk,
                    double wk, double wk1) {
    a.eth[p] = ein + pre / rho;
    a.pregd[p] = (pre - m.pre_bs[p]) * m.GSGAM2[p];
    a.rhogd[p] = (rho - m.rho_bs[p]) * m.GSGAM2[p];
    if (k >= kmin && k <= kmax) {
      double wc = cC.cfact[k] * wk1 + cC.dfact[k] * wk;
      a.vvx[p] = vxk + div_r(wc * gx);
      a.vvy[p] = vyk + div_r(wc * gy);
      a.vvz[p] = vzk + div_r(wc * gz);
    } else {
      a.vvx[p] = 0.0; a.vvy[p] = 0.0; a.vvz[p] = 0.0;
    }
  };
  double pp = 0.0, pr = 0.0, pe = 0.0, px = 0.0, py = 0.0, pz = 0.0, pw = 0.0;   // level k-1
  double rg_prev = 0.0;
  for (int k = 0; k < KA; ++k) {
    int p = c.at(k);
    double RHOG = P[0][p];
    double rho = RHOG / m.GSGAM2[p];
    const auto rr = recip_of(RHOG);   // five quotients by RHOG
    const double vx = div_by(P[1][p], rr), vy = div_by(P[2][p], rr), vz = div_by(P[3][p], rr);
    a.vx[p] = vx;
    a.vy[p] = vy;
    a.vz[p] = vz;
    double ein = div_by(P[5][p], rr);
    double q0 = div_by(a.Pqw[0][p], rr);
    double qd, cv;
    moist_qd_cv([&](int n) { return div_by(a.Pqw[n][p], rr); }, q0, qd, cv);
    double tem = ein / cv;
    const double pre = rho * tem * (qd * cC.Rdry + q0 * cC.Rvap);
    a.tem[p] = tem;
    a.pre[p] = pre;
    a.rho[p] = rho;
    a.ein[p] = ein;
    double w = 0.0;
    if (k >= kmin + 1 && k <= kmax) {
      w = P[4][p] / (mc(m.C2W, c, 0, 2, k) * RHOG + mc(m.C2W, c, 1, 2, k) * rg_prev);
      a.w[p] = w;
    }
    if (k - 1 >= kmin + 1 && k - 1 <= kmax - 1) finish(k - 1, c.at(k - 1), pp, pr, pe, px, py, pz, pw, w);
    pp = pre; pr = rho; pe = ein; px = vx; py = vy; pz = vz; pw = w;
    rg_prev = RHOG;
  }
  // ---- boundary conditions: TEM top/bottom, FREE top, RIGID bottom
  const int pT = c.at(kmax + 1), pK = c.at(kmax), pKm = c.at(kmax - 1);
  const int pB = c.at(kmin - 1), pN = c.at(kmin), pNp = c.at(kmin + 1);
  double tem_top = a.tem[pK];
  double tem_btm = a.tem[pN];
  double pre_top = a.pre[pKm] - a.rho[pK] * (m.PHI[pT] - m.PHI[pKm]);
  double pre_btm = a.pre[pNp] - a.rho[pN] * (m.PHI[pB] - m.PHI[pNp]);
  double rho_top = pre_top / (cC.Rdry * tem_top);
  double rho_btm = pre_btm / (cC.Rdry * tem_btm);
  a.tem[pT] = tem_top; a.tem[pB] = tem_btm;
  a.pre[pT] = pre_top; a.pre[pB] = pre_btm;
  a.rho[pT] = rho_top; a.rho[pB] = rho_btm;
  double rgT = rho_top * m.GSGAM2[pT];
  double rgB = rho_btm * m.GSGAM2[pB];
  P[0][pT] = rgT; P[0][pB] = rgB;
  double einT = cC.CVdry * tem_top, einB = cC.CVdry * tem_btm;
  a.ein[pT] = einT; a.ein[pB] = einB;
  P[5][pT] = rgT * einT; P[5][pB] = rgB * einB;
  double rgK = P[0][pK], rgN = P[0][pN];
  double vT[3], vB[3];
  for (int d = 0; d < 3; ++d) {
    vT[d] = 1.0 * (P[1 + d][pK] / rgK) * rgT;
    vB[d] = -1.0 * (P[1 + d][pN] / rgN) * rgB;
    P[1 + d][pT] = vT[d];
    P[1 + d][pB] = vB[d];
  }
  R* dv[3] = {a.vx, a.vy, a.vz};
  for (int d = 0; d < 3; ++d) {
    dv[d][pT] = P[1 + d][pT] / P[0][pT];
    dv[d][pB] = P[1 + d][pB] / P[0][pB];
  }
  const int kT = kmax + 1;
  double rwT = -(mc(m.C2WGz, c, 0, 6, kT) * vT[0] + mc(m.C2WGz, c, 1, 6, kT) * P[1][pK] +
                 mc(m.C2WGz, c, 2, 6, kT) * vT[1] + mc(m.C2WGz, c, 3, 6, kT) * P[2][pK] +
                 mc(m.C2WGz, c, 4, 6, kT) * vT[2] + mc(m.C2WGz, c, 5, 6, kT) * P[3][pK]);
  P[4][pT] = rwT;
  P[4][pN] = 0.0;
  P[4][pB] = 0.0;
  a.w[pT] = rwT / (mc(m.C2W, c, 0, 2, kT) * rgT + mc(m.C2W, c, 1, 2, kT) * rgK);
  a.w[pN] = P[4][pN] / (mc(m.C2W, c, 0, 2, kmin) * rgN + mc(m.C2W, c, 1, 2, kmin) * rgB);
  a.w[pB] = 0.0;
  // ---- the levels next to the boundary rows
  const int rest[4] = {kmin - 1, kmin, kmax, kmax + 1};
  for (int r = 0; r < 4; ++r) {
    const int k = rest[r];
    const int p = c.at(k);
    const double wk1 = (k >= kmin && k <= kmax) ? a.w[c.at(k + 1)] : 0.0;
    finish(k, p, a.pre[p], a.rho[p], a.ein[p], a.vx[p], a.vy[p], a.vz[p], a.w[p], wk1);
  }
}

// eight 128-thread blocks per SM (64 registers): measured faster than the
// uncapped 84 registers
template <class R>
__global__ void __launch_bounds__(128, NC_MINB(R, 8, NC_F32_DIAG)) k_diag(DiagArgs<R> a, int pole) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l, g, lp;
  if (!map_col(pole, t, i, j, l, g, lp)) return;
  if (!pole) {
    diag_column_fused(col_reg(i, j, l), met_of<R>(false), a, (double)P2(CG.GRD_x, 0, i, j, l),
                      (double)P2(CG.GRD_x, 1, i, j, l), (double)P2(CG.GRD_x, 2, i, j, l));
  } else {
    const R* X = CG.GRD_x_pl;
    diag_column(col_pl(g, lp), met_of<R>(true), a, (double)X[(g * cD.LP + lp) * 3 + 0],
                (double)X[(g * cD.LP + lp) * 3 + 1], (double)X[(g * cD.LP + lp) * 3 + 2]);
  }
}

// ---------------------------------------------------------------------------
// Momentum advection convergence + Coriolis + horizontalize
// (mod_src.py:96-497, kernels/advconv.py:42-108, fluxconv.py:111-208,
// advconvmom.py:111-194).  Outputs grhogv{x,y,z}, grhogw.
// ---------------------------------------------------------------------------
template <class R>
struct AdvMomArgs {
  const R *rg, *rvx, *rvy, *rvz, *rw;    // PROG (post BNDCND)
  const R *vvx, *vvy, *vvz;              // merged velocity
  R *gvx, *gvy, *gvz, *gw;               // out
};

// Tiled momentum advection for interior cells: one block per 32x8 tile of a
// region, marching upward over kmin..kmax (the vertical-momentum tendency at k
// needs the projection at k-1, and the half-level flux at k is reused from the
// level below).  Per level the haloed tile of rhogv, the merged velocity and
// RGAM is staged in shared memory for the three 7-point divergences.  Halo
// cells and boundary levels are not written (their values are never read:
// the large-step tendencies derived from them are replaced by the exchanges).
// Arithmetic and association order are those of the reference's expressions
// (kernels/advconv.py, kernels/advconvmom.py), as in the pole kernel.
template <class R>
__global__ void __launch_bounds__(256, NC_MINB(R, 2, NC_F32_ADVMOM)) k_advmom_t(AdvMomArgs<R> a) {
  constexpr int TXD = 32, TYD = 8;
  constexpr int PX = TXD + 2, PY = TYD + 2;
  __shared__ R s_rv[3][PY * PX], s_vv[3][PY * PX], s_rg[PY * PX];
  const int ntx = (cD.G - 2 + TXD - 1) / TXD;
  const int l = (int)blockIdx.z;
  const int i0 = 1 + ((int)blockIdx.x % ntx) * TXD, j0 = 1 + ((int)blockIdx.x / ntx) * TYD;
  const int G = cD.G, gmax = cD.G - 2, kmin = cD.kmin, kmax = cD.kmax;
  const int tid = threadIdx.x, tx = tid % TXD, ty = tid / TXD;
  const int i = i0 + tx, j = j0 + ty;
  const bool own = (i <= gmax) && (j <= gmax);
  const R* rv[3] = {a.rvx, a.rvy, a.rvz};
  const R* vv[3] = {a.vvx, a.vvy, a.vvz};
  const R* cz = CG.C2WGz;
  const int n = cD.npti;
  R gx = R(0.0), gy = R(0.0), gz = R(0.0);
  int q0 = 0;
  if (own) {
    gx = div_r(P2(CG.GRD_x, 0, i, j, l));
    gy = div_r(P2(CG.GRD_x, 1, i, j, l));
    gz = div_r(P2(CG.GRD_x, 2, i, j, l));
    q0 = ix(i, j, 0, l);
  }
  R vmh_lo[3] = {R(0.0), R(0.0), R(0.0)};
  R gwc_prev = R(0.0);
  for (int k = kmin; k <= kmax; ++k) {
    for (int p = tid; p < PX * PY; p += blockDim.x) {
      const int ii = i0 - 1 + p % PX, jj = j0 - 1 + p / PX;
      const bool ok = ii < G && jj < G;
      const int q = ok ? ix(ii, jj, k, l) : 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        s_rv[d][p] = ok ? rv[d][q] : R(0.0);
        s_vv[d][p] = ok ? vv[d][q] : R(0.0);
      }
      s_rg[p] = ok ? gam_at(CG.RGAM, q) : R(0.0);
    }
    __syncthreads();
    if (own) {
      const int c0 = (ty + 1) * PX + (tx + 1);
      const int nb[7] = {c0, c0 + 1, c0 + PX + 1, c0 + PX, c0 - 1, c0 - PX - 1, c0 - PX};
      const int p = q0 + k * cD.planei;
      const int kk = k + 1;
      const bool hv = (kk > kmin && kk <= kmax);
      const int qh = p + cD.planei;   // level k+1 of the own column
      R dv[3];
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        R acc[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          R sm = R(0.0);
#pragma unroll
          for (int m = 0; m < 7; ++m) {
            const R v = (s_rv[d][nb[m]] * s_vv[s][nb[m]]) * s_rg[nb[m]];
            const R t = P2(CG.coef_div, d * 7 + m, i, j, l) * v;
            sm = (m == 0) ? t : sm + t;
          }
          acc[d] = sm;
        }
        const R div = acc[0] + acc[1] + acc[2];
        R vmh_hi = R(0.0);
        if (hv) {
          const R sh = vv[s][qh], sl = s_vv[s][c0];
          const R h = cz[qh] * (rv[0][qh] * sh) + cz[n + qh] * (s_rv[0][c0] * sl) +
                           cz[2 * n + qh] * (rv[1][qh] * sh) + cz[3 * n + qh] * (s_rv[1][c0] * sl) +
                           cz[4 * n + qh] * (rv[2][qh] * sh) + cz[5 * n + qh] * (s_rv[2][c0] * sl);
          const R sw = a.rw[qh] * (CC.afact[kk] * sh + CC.bfact[kk] * sl);
          vmh_hi = h * gam_at(CG.RGAMH, qh) + R(1.0) * sw * CG.RGSQRTH[qh];
        }
        dv[s] = -div - (vmh_hi - vmh_lo[s]) * CC.rdgz[k];
        vmh_lo[s] = vmh_hi;
      }
      const R rh = a.rg[p];
      const R dvx = dv[0] - (-R(2.0) * rh * (CC.OHM * s_vv[1][c0]));
      const R dvy = dv[1] - (R(2.0) * rh * (CC.OHM * s_vv[0][c0]));
      const R dvz = dv[2];
      const R prd = dvx * gx + dvy * gy + dvz * gz;
      a.gvx[p] = dvx - prd * gx;
      a.gvy[p] = dvy - prd * gy;
      a.gvz[p] = dvz - prd * gz;
      const R gwc = prd * CC.alpha;
      a.gw[p] = (k >= kmin + 1) ? (CG.C2W[p] * gwc + CG.C2W[n + p] * gwc_prev) : R(0.0);
      gwc_prev = gwc;
    }
    __syncthreads();
  }
}

// pole part of the momentum advection (one thread per pole column (g, lp))
template <class R>
__device__ R advconv_pl_at(int g, int lp, int k, const Col& c, const MetT<R>& m, const R* rvx,
                                const R* rvy, const R* rvz, const R* rw, const R* scl) {
  R div = R(0.0);
  if (g == 0) {
    const R* cd = CG.coef_div_pl;
    R row = R(0.0);
    for (int v = 0; v < 6; ++v) {
      int q = ipl(v, k, lp);
      R vx = (rvx[q] * scl[q]) * gam_at(CG.RGAM_pl, q);
      R vy = (rvy[q] * scl[q]) * gam_at(CG.RGAM_pl, q);
      R vz = (rvz[q] * scl[q]) * gam_at(CG.RGAM_pl, q);
      R pv = cd[(v * cD.LP + lp) * 3 + 0] * vx + cd[(v * cD.LP + lp) * 3 + 1] * vy +
                  cd[(v * cD.LP + lp) * 3 + 2] * vz;
      row = (v == 0) ? pv : row + pv;
    }
    div = row;
  }
  auto vmh = [&](int kk) -> R {
    if (kk <= cD.kmin || kk > cD.kmax) return R(0.0);
    R h = vmh_horiz(c, m, kk, [&](int k2, int d) -> R {
      int q = c.at(k2);
      const R* rv = (d == 0) ? rvx : ((d == 1) ? rvy : rvz);
      return rv[q] * scl[q];
    });
    int q = c.at(kk);
    R sw = rw[q] * (CC.afact[kk] * scl[q] + CC.bfact[kk] * scl[c.at(kk - 1)]);
    return h + R(1.0) * sw * m.RGSQRTH[q];
  };
  return -div - (vmh(k + 1) - vmh(k)) * CC.rdgz[k];
}

template <class R>
__global__ void k_advmom_pl(AdvMomArgs<R> a) {
  int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= 6 * cD.LP) return;
  int g = t / cD.LP, lp = t % cD.LP;
  const Col c = col_pl(g, lp);
  const MetT<R> m = met_of<R>(true);
  const R* X = CG.GRD_x_pl;
  const R gx = div_r(X[(g * cD.LP + lp) * 3 + 0]), gy = div_r(X[(g * cD.LP + lp) * 3 + 1]),
               gz = div_r(X[(g * cD.LP + lp) * 3 + 2]);
  R gwc_prev = R(0.0);
  for (int k = 0; k < cD.KA; ++k) {
    int p = c.at(k);
    if (k < cD.kmin || k > cD.kmax) {
      a.gvx[p] = R(0.0); a.gvy[p] = R(0.0); a.gvz[p] = R(0.0); a.gw[p] = R(0.0);
      continue;
    }
    R dv[3];
    const R* vv[3] = {a.vvx, a.vvy, a.vvz};
    for (int s = 0; s < 3; ++s) dv[s] = advconv_pl_at(g, lp, k, c, m, a.rvx, a.rvy, a.rvz, a.rw, vv[s]);
    R rh = a.rg[p];
    R dvx = dv[0] - (-R(2.0) * rh * (CC.OHM * a.vvy[p]));
    R dvy = dv[1] - (R(2.0) * rh * (CC.OHM * a.vvx[p]));
    R dvz = dv[2];
    R prd = dvx * gx + dvy * gy + dvz * gz;
    a.gvx[p] = dvx - prd * gx;
    a.gvy[p] = dvy - prd * gy;
    a.gvz[p] = dvz - prd * gz;
    R gwc = prd * CC.alpha;
    a.gw[p] = (k >= cD.kmin + 1) ? (mc(m.C2W, c, 0, 2, k) * gwc + mc(m.C2W, c, 1, 2, k) * gwc_prev) : R(0.0);
    gwc_prev = gwc;
  }
}

// ---------------------------------------------------------------------------
// Hyperdiffusion (mod_numfilter.py:845-1469, lap_order 2, DIRECT).
// Pass 1: vt = -lap(src), src = (vx, vy, vz, w, tem - tem_bs, rho - rho_bs).
// Pass 2: vt2 = -(lap of comps 0..3, kh-weighted diffusion of comps 4, 5).
// ---------------------------------------------------------------------------
template <class R>
struct Six { const R* f[6]; };
template <class R>
struct SixOut { R* f[6]; };

template <class R>
__global__ void k_hdiff1(Six<R> src, SixOut<R> out) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l;
  if (!col_of(t, i, j, l)) return;
  const bool in = interior(i, j);
  // the column's seven laplacian coefficients, loaded once for all levels
  R cl[7];
#pragma unroll
  for (int m = 0; m < 7; ++m) cl[m] = in ? P2(CG.coef_lap, m, i, j, l) : R(0.0);
  for (int k = 0; k < cD.KA; ++k) {
    int p = ix(i, j, k, l);
#pragma unroll
    for (int n = 0; n < 6; ++n) {
      R v = R(0.0);
      if (in) {
        const R* s = src.f[n];
        const R* bs = (n == 4) ? CG.tem_bs : CG.rho_bs;
        // lap7 (kernels/oprtlaplacian.py:41-55) with the reference-state
        // deviation for TEM and RHO
        auto scl = [&](int m) {
          const int q = ix(i + kNbI[m], j + kNbJ[m], k, l);
          return (n >= 4) ? s[q] - bs[q] : s[q];
        };
        v = cl[0] * scl(0);
#pragma unroll
        for (int m = 1; m < 7; ++m) v = v + cl[m] * scl(m);
      }
      out.f[n][p] = -v;
    }
  }
}

template <class R>
__global__ void k_hdiff1_pl(Six<R> src, SixOut<R> out) {
  int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  int k = t / cD.LP, lp = t % cD.LP;
  for (int n = 0; n < 6; ++n) {
    R row = R(0.0);
    for (int v = 0; v < 6; ++v) {
      int q = ipl(v, k, lp);
      R s = src.f[n][q];
      if (n == 4) s = s - CG.tem_bs_pl[q];
      if (n == 5) s = s - CG.rho_bs_pl[q];
      R tv = CG.coef_lap_pl[v * cD.LP + lp] * s;
      row = (v == 0) ? tv : row + tv;
    }
    out.f[n][ipl(0, k, lp)] = -row;
    for (int g = 1; g < 6; ++g) out.f[n][ipl(g, k, lp)] = -R(0.0);
  }
}

// The three vertex weights of each triangle of the Kh-weighted diffusion,
// formed once from the interpolation coefficients with the reference's
// expressions (kernels/oprtdiffusion.py:59-90): for direction d and triangle
// t (i or j), 2*c1 - c2 - c3, -c1 + 2*c2 - c3 and -c1 - c2 + 2*c3 of
// coef_intp[d][0..2][t].  Planes [((d*3+m)*2+t)][l][j][i].
__global__ void k_intp_weights(const double* ci, double* w, int npt2) {
  const int q = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (q >= npt2) return;
  for (int d = 0; d < 3; ++d)
    for (int t = 0; t < 2; ++t) {
      const double c1 = ci[((d * 3 + 0) * 2 + t) * npt2 + q], c2 = ci[((d * 3 + 1) * 2 + t) * npt2 + q];
      const double c3 = ci[((d * 3 + 2) * 2 + t) * npt2 + q];
      w[((d * 3 + 0) * 2 + t) * npt2 + q] = 2.0 * c1 - c2 - c3;
      w[((d * 3 + 1) * 2 + t) * npt2 + q] = -c1 + 2.0 * c2 - c3;
      w[((d * 3 + 2) * 2 + t) * npt2 + q] = -c1 - c2 + 2.0 * c3;
    }
}

#define HD_DX 32
#define HD_DY 8

// Kh of the hyperdiffusion at level k: the uniform DIRECT coefficient, or for
// NONLINEAR1 (mod_numfilter.py:1153-1184) the coefficient from the
// temperature-deviation Laplacian lapT of the first pass,
// clip(2 AREA^2 / dtl * (|lapT| / 300 * AREA), Kh_coef_minlim, kh_max(k))
template <class R>
__device__ __forceinline__ R hdiff_kh(R lapT, int k) {
  if (!CC.hdiff_nl) return CC.Kh;
  const R c = CC.nl_c1 * (fabs(lapT) / R(300.0) * CC.nl_area);
  return fmin(fmax(c, CC.nl_min), CC.nl_khmax[k]);
}

// Second hyperdiffusion pass, one block per (HD_NK levels, HD_DX x HD_DY tile)
// of interior cells: the haloed tile of the six Laplacians and of rhog is
// staged in shared memory per level, the triangle gradients of the
// temperature and density Laplacians are formed once (with the singular-point
// fix at the (0,0) vertex), then each thread writes its cell's four
// Laplacians and two Kh-weighted diffusions (kernels/oprtlaplacian.py:41-55,
// kernels/oprtdiffusion.py).  Halo cells are left to the exchange that
// follows.  The tile's k-independent triangle weights (intp_w, 18 planes) are
// staged in shared memory and the cell's Laplacian and diffusion coefficients
// (coef_lap 7, coef_diff 18) held in registers once for all of the block's
// levels, instead of re-read from L2 at every level.  Dynamic shared memory:
// hdiff2_m_smem<R>() bytes (45 KB float, 90 KB double).  Kh per cell from
// hdiff_kh (the first pass's temperature Laplacian is the staged field 4).
#ifndef HD_NK
#define HD_NK 6
#endif
template <class R>
constexpr int hdiff2_m_smem() {
  return ((18 + 12) * (HD_DX + 1) * (HD_DY + 1) + 7 * (HD_DX + 2) * (HD_DY + 2)) * (int)sizeof(R);
}
template <class R>
__global__ void __launch_bounds__(HD_DX * HD_DY, NC_MINB(R, 2, 4)) k_hdiff2_m(Six<R> vt, const R* rhog,
                                                                            SixOut<R> out) {
  constexpr int PX = HD_DX + 2, PY = HD_DY + 2, NP = PX * PY, TX = HD_DX + 1, TY = HD_DY + 1, NT = TX * TY;
  extern __shared__ __align__(16) unsigned char hd_smem[];
  R* s_w = reinterpret_cast<R*>(hd_smem);   // [18][NT] triangle weights
  R* s_f = s_w + 18 * NT;                     // [6][NP] the six Laplacians
  R* s_r = s_f + 6 * NP;                      // [NP] rhog
  R* s_t = s_r + NP;                          // [2][6][NT] triangle values of fields 4 and 5
  const int l = (int)blockIdx.z;
  const int ntx = (cD.G - 2 + HD_DX - 1) / HD_DX;
  const int i0 = 1 + ((int)blockIdx.y % ntx) * HD_DX, j0 = 1 + ((int)blockIdx.y / ntx) * HD_DY;
  const int k0 = (int)blockIdx.x * HD_NK, k1 = min(k0 + HD_NK, cD.KA);
  const int G = cD.G, gmax = cD.G - 2;
  const int tid = threadIdx.x, tx = tid % HD_DX, ty = tid / HD_DX;
  const int i = i0 + tx, j = j0 + ty;
  const bool own = (i <= gmax) && (j <= gmax);
  const R kfac[2] = {CC.CVdry, CC.hdiff_fact_rho};
  for (int p = tid; p < NT; p += blockDim.x) {
    const int ii = i0 - 1 + p % TX, jj = j0 - 1 + p / TX;
    const bool ok = ii <= G - 2 && jj <= G - 2;
#pragma unroll
    for (int m = 0; m < 18; ++m) s_w[m * NT + p] = ok ? P2(CG.intp_w, m, ii, jj, l) : R(0.0);
  }
  R cl[7], cd[18];
  if (own) {
#pragma unroll
    for (int m = 0; m < 7; ++m) cl[m] = P2(CG.coef_lap, m, i, j, l);
#pragma unroll
    for (int m = 0; m < 18; ++m) cd[m] = P2(CG.coef_diff, m, i, j, l);
  }
  for (int k = k0; k < k1; ++k) {
    for (int p = tid; p < NP; p += blockDim.x) {
      const int ii = i0 - 1 + p % PX, jj = j0 - 1 + p / PX;
      const bool ok = ii < G && jj < G;
      const int q = ok ? ix(ii, jj, k, l) : 0;
#pragma unroll
      for (int n = 0; n < 6; ++n) s_f[n * NP + p] = ok ? vt.f[n][q] : R(0.0);
      s_r[p] = ok ? rhog[q] : R(0.0);
    }
    __syncthreads();
    for (int p = tid; p < NT; p += blockDim.x) {
      const int px = p % TX, py = p / TX;
      const int ii = i0 - 1 + px, jj = j0 - 1 + py;
      const bool ok = ii <= G - 2 && jj <= G - 2;
      const int ia = py * PX + px, ib = ia + 1, ic = ia + PX + 1, id = ia + PX;
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        const R* sf = s_f + (4 + f) * NP;
        const R s0 = sf[ia], sip = sf[ib], sd = sf[ic], sjp = sf[id];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          R ti = R(0.0), tj = R(0.0);
          if (ok) {
            // weights 2c1-c2-c3, -c1+2c2-c3, -c1-c2+2c3 of the i and j triangles (k_intp_weights)
            const R w1i = s_w[((d * 3 + 0) * 2 + 0) * NT + p], w2i = s_w[((d * 3 + 1) * 2 + 0) * NT + p];
            const R w3i = s_w[((d * 3 + 2) * 2 + 0) * NT + p], w1j = s_w[((d * 3 + 0) * 2 + 1) * NT + p];
            const R w2j = s_w[((d * 3 + 1) * 2 + 1) * NT + p], w3j = s_w[((d * 3 + 2) * 2 + 1) * NT + p];
            ti = div3(w1i * s0 + w2i * sip + w3i * sd);
            tj = div3(w1j * s0 + w2j * sd + w3j * sjp);
          }
          s_t[(f * 6 + d) * NT + p] = ti;
          s_t[(f * 6 + 3 + d) * NT + p] = tj;
        }
      }
    }
    __syncthreads();
    if (i0 == 1 && j0 == 1 && tid < 6) {   // singular-point fix of the (0,0) triangle, fields 4 and 5
      const int f = tid / 3, d = tid % 3;
      const R m0 = (R)CG.pntmask[l * 2 + 0], m1 = (R)CG.pntmask[l * 2 + 1];
      s_t[(f * 6 + d) * NT] = s_t[(f * 6 + d) * NT] * m0 + s_t[(f * 6 + 3 + d) * NT + 1] * m1;
    }
    __syncthreads();
    if (own) {
      const int q = ix(i, j, k, l);
      const int c0 = (ty + 1) * PX + (tx + 1);
      const int nb[7] = {c0, c0 + 1, c0 + PX + 1, c0 + PX, c0 - 1, c0 - PX - 1, c0 - PX};
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        const R* sf = s_f + n * NP;
        R v = cl[0] * sf[nb[0]];
#pragma unroll
        for (int m = 1; m < 7; ++m) v = v + cl[m] * sf[nb[m]];
        out.f[n][q] = -v;
      }
      const int ta = (ty + 1) * TX + (tx + 1), tb = ta - 1, tc = ta - TX - 1, td = ta - TX;
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        auto kh = [&](int pt) { return s_r[pt] * kfac[f] * hdiff_kh<R>(s_f[4 * NP + pt], k); };
        const R kh0 = kh(nb[0]);
        const R kf1 = R(0.5) * (kh0 + kh(nb[2])), kf2 = R(0.5) * (kh0 + kh(nb[3])), kf3 = R(0.5) * (kh0 + kh(nb[4]));
        const R kf4 = R(0.5) * (kh0 + kh(nb[5])), kf5 = R(0.5) * (kh0 + kh(nb[6])), kf6 = R(0.5) * (kh0 + kh(nb[1]));
        R inner = R(0.0);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const R* ti = s_t + (f * 6 + d) * NT;
          const R* tj = s_t + (f * 6 + 3 + d) * NT;
          const R aTI = ti[ta], aTJ = tj[ta], bTI = ti[tb];
          const R cTI = ti[tc], cTJ = tj[tc], dTJ = tj[td];
          const R blk = kf1 * cd[d * 6 + 0] * (aTI + aTJ) + kf2 * cd[d * 6 + 1] * (aTJ + bTI) +
                        kf3 * cd[d * 6 + 2] * (bTI + cTJ) + kf4 * cd[d * 6 + 3] * (cTJ + cTI) +
                        kf5 * cd[d * 6 + 4] * (cTI + dTJ) + kf6 * cd[d * 6 + 5] * (dTJ + aTI);
          inner = (d == 0) ? blk : inner + blk;
        }
        out.f[4 + f][q] = -inner;
      }
    }
    __syncthreads();
  }
}

template <class R>
__global__ void k_hdiff2_pl(Six<R> vt, const R* rhog, SixOut<R> out) {
  int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  int k = t / cD.LP, lp = t % cD.LP;
  for (int n = 0; n < 6; ++n) {
    const R* s = vt.f[n];
    R row = R(0.0);
    if (n < 4) {
      for (int v = 0; v < 6; ++v) {
        R tv = CG.coef_lap_pl[v * cD.LP + lp] * s[ipl(v, k, lp)];
        row = (v == 0) ? tv : row + tv;
      }
    } else {
      // kernels/oprtdiffusion.py:137-177
      const R fac = (n == 4) ? CC.CVdry : CC.hdiff_fact_rho;
      R sn = s[ipl(0, k, lp)];
      R vt_[5][3];
      for (int v = 1; v <= 5; ++v) {
        int vp1 = (v == 5) ? 1 : v + 1;
        R sij = s[ipl(v, k, lp)], sp1 = s[ipl(vp1, k, lp)];
        for (int d = 0; d < 3; ++d) {
          const R* cI = CG.coef_intp_pl + ((v * cD.LP + lp) * 3 + d) * 3;
          R c0 = cI[0], c1 = cI[1], c2 = cI[2];
          vt_[v - 1][d] = div3((R(2.0) * c0 - c1 - c2) * sn + (-c0 + R(2.0) * c1 - c2) * sij + (-c0 - c1 + R(2.0) * c2) * sp1);
        }
      }
      R khn = rhog[ipl(0, k, lp)] * fac * hdiff_kh<R>(vt.f[4][ipl(0, k, lp)], k);
      for (int v = 1; v <= 5; ++v) {
        int vm1 = (v == 1) ? 5 : v - 1;
        R khv = rhog[ipl(v, k, lp)] * fac * hdiff_kh<R>(vt.f[4][ipl(v, k, lp)], k);
        R kavg = R(0.5) * (khn + khv);
        R sd = R(0.0);
        for (int d = 0; d < 3; ++d) {
          R cdv = CG.coef_diff_pl[(v * cD.LP + lp) * 3 + d];
          R tv = cdv * (vt_[vm1 - 1][d] + vt_[v - 1][d]);
          sd = (d == 0) ? tv : sd + tv;
        }
        R contrib = kavg * sd;
        row = (v == 1) ? contrib : row + contrib;
      }
    }
    out.f[n][ipl(0, k, lp)] = -row;
    for (int g = 1; g < 6; ++g) out.f[n][ipl(g, k, lp)] = -R(0.0);
  }
}

// ---------------------------------------------------------------------------
// Large-step tendency: hyperdiffusion tendency (mod_numfilter.py:1519-1578)
// + horizontalize (mod_numfilter.py:1364-1369) + g_TEND = adv + f
// (mod_dynamics.py:1340-1464).  All columns; projection on interior points.
// ---------------------------------------------------------------------------
template <class R>
struct GtendArgs {
  Six<R> vt2;                       // post-COMM hyperdiffusion Laplacians
  const R* lapT;                    // the first pass's temperature Laplacian (NONLINEAR1 Kh)
  const R *vx, *vy, *vz, *w;        // diagnosed velocities (Rayleigh sponge)
  const R *rhog, *gvx, *gvy, *gvz, *gw;
  R* gT0[6];
  R* frhog;                 // f_TEND[RHOG] (tracer input)
};

template <class R>
__device__ void gtend_column(const Col c, const MetT<R> m, const GtendArgs<R>& a, int i, int j, int l, int g, int lp) {
  for (int k = 0; k < cD.KA; ++k) {
    int p = c.at(k);
    R rg = a.rhog[p];
    R rgh = R(0.0);
    if (k >= cD.kmin) rgh = mc(m.C2W, c, 0, 2, k) * rg + mc(m.C2W, c, 1, 2, k) * a.rhog[c.at(k - 1)];
    const R Kh = hdiff_kh<R>(CC.hdiff_nl ? a.lapT[p] : R(0.0), k);
    // the coefficient of w: Kh itself (DIRECT), or for NONLINEAR1 the average of
    // levels k and k-1 on kmin+1..kmax and zero elsewhere (mod_numfilter.py:1186-1206)
    R Khh = Kh;
    if (CC.hdiff_nl)
      Khh = (k > cD.kmin && k <= cD.kmax) ? R(0.5) * (Kh + hdiff_kh<R>(a.lapT[c.at(k - 1)], k - 1)) : R(0.0);
    R fx = -(a.vt2.f[0][p] * Kh + R(0.0)) * rg;
    R fy = -(a.vt2.f[1][p] * Kh + R(0.0)) * rg;
    R fz = -(a.vt2.f[2][p] * Kh + R(0.0)) * rg;
    R fw = -(a.vt2.f[3][p] * Khh + R(0.0)) * rgh;
    R fe = -(a.vt2.f[4][p] + R(0.0));
    R fr = -(a.vt2.f[5][p] + R(0.0));
    if (!c.pole) {
      if (interior(i, j)) horiz_reg(i, j, l, fx, fy, fz);
    } else {
      horiz_pl(g, lp, fx, fy, fz);
    }
    if (CC.rayleigh) {   // the sponge on the hyperdiffusion tendency (mod_numfilter.py:240-271)
      if (!CC.rayleigh_only_w) {
        const R coef = CC.ray_c[k] * rg;
        fx = fx - coef * a.vx[p];
        fy = fy - coef * a.vy[p];
        fz = fz - coef * a.vz[p];
      }
      const R rgm1 = k > 0 ? a.rhog[c.at(k - 1)] : R(0.0);
      fw = fw - CC.ray_ch[k] * a.w[p] * (mc(m.C2W, c, 0, 2, k) * rg + mc(m.C2W, c, 1, 2, k) * rgm1);
    }
    a.gT0[0][p] = R(0.0) + fr;
    a.gT0[1][p] = a.gvx[p] + fx;
    a.gT0[2][p] = a.gvy[p] + fy;
    a.gT0[3][p] = a.gvz[p] + fz;
    a.gT0[4][p] = a.gw[p] + fw;
    a.gT0[5][p] = R(0.0) + fe;
    a.frhog[p] = fr;
  }
}

template <class R>
__global__ void k_gtend(GtendArgs<R> a, int pole) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l, g, lp;
  if (!map_col(pole, t, i, j, l, g, lp)) return;
  if (!pole) gtend_column(col_reg(i, j, l), met_of<R>(false), a, i, j, l, 0, 0);
  else gtend_column(col_pl(g, lp), met_of<R>(true), a, 0, 0, 0, g, lp);
}

}  // namespace nc
