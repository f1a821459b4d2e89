// Tracer advection of the last RK stage: MIURA2004 horizontal scheme with
// the Thuburn horizontal and vertical flux limiters, Strang-split V/H/V
// (pynicamdc/nhm/dynamics/mod_src_tracer.py:83-1228).
#pragma once
#include "nc_small.cuh"

namespace nc {

// ---------------------------------------------------------------------------
// tracer-independent part of the first vertical step (kernels/tracervertflux.py)
// flx_v and the updated density rhog_t, on every column.
// ---------------------------------------------------------------------------
template <class R>
struct TrcFluxArgs {
  const R *rvx, *rvy, *rvz, *rw;    // time-mean momentum (PROG_mean)
  const R* rhog_in;                 // density at the start of the step
  const R* frhog;
  R *flx_v, *rhog_t;
  R dt;
};

template <class R>
__device__ void trc_vflux_column(const Col c, const MetT<R> m, const TrcFluxArgs<R>& a) {
  const int KA = cD.KA, kmin = cD.kmin, kmax = cD.kmax;
  for (int k = 0; k < KA; ++k) {
    int p = c.at(k);
    R f = R(0.0);
    if (k >= kmin + 1 && k <= kmax) {
      int pm = c.at(k - 1);
      R horiz = (mc(m.C2WGz, c, 0, 6, k) * a.rvx[p] + mc(m.C2WGz, c, 1, 6, k) * a.rvx[pm] +
                      mc(m.C2WGz, c, 2, 6, k) * a.rvy[p] + mc(m.C2WGz, c, 3, 6, k) * a.rvy[pm] +
                      mc(m.C2WGz, c, 4, 6, k) * a.rvz[p] + mc(m.C2WGz, c, 5, 6, k) * a.rvz[pm]) * gam_at(m.RGAMH, p);
      R vert = a.rw[p] * m.RGSQRTH[p];
      f = (horiz + vert) * R(0.5) * a.dt;
    }
    a.flx_v[p] = f;
  }
  for (int k = 0; k < KA; ++k) {
    int p = c.at(k);
    R r = R(0.0);
    if (k >= kmin && k <= kmax) {
      r = a.rhog_in[p] - (a.flx_v[c.at(k + 1)] - a.flx_v[p]) * CC.rdgz[k] + R(0.0) * a.frhog[p] * a.dt;
    } else if (k == kmin - 1) {
      r = a.rhog_in[c.at(kmin)];
    } else if (k == kmax + 1) {
      r = a.rhog_in[c.at(kmax)];
    }
    a.rhog_t[p] = r;
  }
}

template <class R>
__global__ void k_trc_vflux(TrcFluxArgs<R> a, int pole) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l, g, lp;
  if (!map_col(pole, t, i, j, l, g, lp)) return;
  if (!pole) trc_vflux_column(col_reg(i, j, l), met_of<R>(false), a);
  else trc_vflux_column(col_pl(g, lp), met_of<R>(true), a);
}

// ---------------------------------------------------------------------------
// one vertical fractional step of one tracer with the vertical Thuburn
// limiter (mod_src_tracer.py:389-533 and 1036-1204, limiter :1909-2074)
// ---------------------------------------------------------------------------
template <class R>
struct TrcVadvArgs {
  R* rhogq;
  const R *den, *flx_v, *frhog;
  R dt, bcoef;      // d = bcoef*frhog/den*dt
  int clamp;             // second step: zero tiny negatives, then add dt*0
  R dtl;
};

// One upward sweep with the values of levels k-1, k, k+1 in registers: at
// level k the cell's outflow bounds are formed, the face value qh[k] is
// limited with the bounds of cells k-1 and k, and cell k-1, whose two faces
// are then final, is updated.  The same expressions as the three-pass form
// of the reference (q, qh and ck on every level, the limiter, the update),
// in the same order, so the same results.
template <class R>
__device__ void trc_vadv_column(const Col c, const TrcVadvArgs<R>& a) {
  const int KA = cD.KA, kmin = cD.kmin, kmax = cD.kmax;
  const R BIG = CC.HUGE_, EPS = CC.EPS;
  auto finish = [&](int k, R x) {   // clamp and store of one updated level
    if (a.clamp && x > -R(1.0e-10) && x < R(0.0)) x = R(0.0);
    if (a.clamp) x = x + a.dtl * R(0.0);
    a.rhogq[c.at(k)] = x;
  };
  // q at kmin-1 and kmin, den and flx_v at kmin (read before the ghost levels are zeroed)
  const int p = c.at(kmin);
  R rq_m = a.rhogq[c.at(kmin - 1)], rq_k = a.rhogq[p];
  R q_m = rq_m / __ldg(&a.den[c.at(kmin - 1)]), q_k = rq_k / __ldg(&a.den[p]);
  R den_k = __ldg(&a.den[p]), flx_k = __ldg(&a.flx_v[p]);
  R qmin_prev = R(0.0), qmax_prev = R(0.0), qh_prev = R(0.0), rq_prev = R(0.0), flx_prev = R(0.0);
  for (int k = kmin; k <= kmax; ++k) {
    const int pp = c.at(k + 1);
    const R rq_p = a.rhogq[pp], den_p = __ldg(&a.den[pp]), flx_p = __ldg(&a.flx_v[pp]);
    const R q_p = rq_p / den_p;
    const R ck0 = -flx_k / den_k * CC.rdgz[k];
    const R ck1 = flx_p / den_k * CC.rdgz[k];
    const R ck0_p = (k + 1 <= kmax) ? -flx_p / den_p * CC.rdgz[k + 1] : R(0.0);
    const R qh_raw = CC.afact[k] * q_k + CC.bfact[k] * q_m;
    const R inL = R(0.5) - copysign(R(0.5), ck0);
    const R inU = R(0.5) + copysign(R(0.5), ck0_p);
    const R qc = q_k, qb = q_m, qa = q_p;
    const R QminL = (inL == R(1.0)) ? npmin(qc, qb) : BIG;
    const R QminU = (inU == R(1.0)) ? npmin(qc, qa) : BIG;
    const R QmaxL = (inL == R(1.0)) ? npmax(qc, qb) : -BIG;
    const R QmaxU = (inU == R(1.0)) ? npmax(qc, qa) : -BIG;
    const R qnmin = npmin(npmin(QminL, QminU), qc);
    const R qnmax = npmax(npmax(QmaxL, QmaxU), qc);
    const R c1 = ck0, c2 = ck1;
    const R Cin = inL * c1 + inU * c2;
    const R Cout = (R(1.0) - inL) * c1 + (R(1.0) - inU) * c2;
    const R CQmin = inL * c1 * QminL + inU * c2 * QminU;
    const R CQmax = inL * c1 * QmaxL + inU * c2 * QmaxU;
    const R zsw = R(0.5) - copysign(R(0.5), fabs(Cout) - EPS);
    const R dk = a.bcoef * __ldg(&a.frhog[c.at(k)]) / den_k * a.dt;
    const R qomin = ((qc - qnmax) + qnmax * (Cin + Cout - dk) - CQmax) / (Cout + zsw) * (R(1.0) - zsw) + qc * zsw;
    const R qomax = ((qc - qnmin) + qnmin * (Cin + Cout - dk) - CQmin) / (Cout + zsw) * (R(1.0) - zsw) + qc * zsw;
    R qh = R(0.0);   // the face at kmin stays zero
    if (k > kmin)
      qh = inL * npmin(npmax(qh_raw, qmin_prev), qmax_prev) + (R(1.0) - inL) * npmin(npmax(qh_raw, qomin), qomax);
    if (k > kmin) finish(k - 1, rq_prev - (flx_k * qh - flx_prev * qh_prev) * CC.rdgz[k - 1]);
    qmin_prev = qomin;
    qmax_prev = qomax;
    qh_prev = qh;
    rq_prev = rq_k;
    flx_prev = flx_k;
    q_m = q_k; q_k = q_p; rq_k = rq_p;
    den_k = den_p; flx_k = flx_p;
  }
  // cell kmax: its upper face (kmax+1) is zero
  finish(kmax, rq_prev - (flx_k * R(0.0) - flx_prev * qh_prev) * CC.rdgz[kmax]);
  for (int k = 0; k < kmin; ++k) finish(k, R(0.0));
  for (int k = kmax + 1; k < KA; ++k) finish(k, R(0.0));
}

template <class R>
__global__ void k_trc_vadv(TrcVadvArgs<R> a, int pole) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l, g, lp;
  if (!map_col(pole, t, i, j, l, g, lp)) return;
  if (!pole) trc_vadv_column(col_reg(i, j, l), a);
  else trc_vadv_column(col_pl(g, lp), a);
}

// ---------------------------------------------------------------------------
// horizontal mass flux through the six hexagon edges and the upwind mass
// centroids (mod_src_tracer.py:1376-1484), Courant numbers and the upwind
// mask (mod_src_tracer.py:716-718)
// ---------------------------------------------------------------------------
template <class R>
struct TrcHfluxArgs {
  const R *rho, *rvx, *rvy, *rvz;   // PROG_mean rhog and momentum (times RGAM on the fly)
  const R* rhog_t;
  R* flx[6];
  R* xc[9];                          // face*3 + dir (AI, AIJ, AJ)
  R* ch[6];
  R* cm[6];
  R dt;
};

// flux and centroid of face f of cell (ii,jj) given the summed vertex values
template <class R>
__device__ __forceinline__ R trc_face(const TrcHfluxArgs<R>& a, int ii, int jj, int l, int f, const R s[4],
                                           R xc[3]) {
  R rr2 = R(1.0) / npmax(s[0], CC.EPS);
  R flux = R(0.5) * (s[1] * P2c(CG.GMTR_a, f * 3 + 0, ii, jj, l) + s[2] * P2c(CG.GMTR_a, f * 3 + 1, ii, jj, l) +
                       s[3] * P2c(CG.GMTR_a, f * 3 + 2, ii, jj, l));
  for (int d = 0; d < 3; ++d) xc[d] = P2c(CG.GRD_xr, f * 3 + d, ii, jj, l) - s[1 + d] * rr2 * a.dt * R(0.5);
  return flux;
}

// One block per level and 32 x 8 tile of cells, the halo ring included (every
// cell gets its six faces; a face the reference leaves out is zero): rho and
// rho*v*RGAM of the haloed tile staged in shared memory, the triangle values
// TI/TJ of every vertex the tile's faces use formed once
// (mod_src_tracer.py:1390-1412, the singular-point fix at the (0,0) vertex
// after them), then each cell's faces 0..2 and its neighbours' faces 0..2
// (its faces 3..5, opposite sign) from those, with the face coefficients of
// the face's owner cell (mod_src_tracer.py:1414-1484).
#define TH_DX 32
#define TH_DY 8
template <class R>
__global__ void __launch_bounds__(TH_DX * TH_DY) k_trc_hflux_t(TrcHfluxArgs<R> a) {
  constexpr int PX = TH_DX + 2, PY = TH_DY + 2, TX = TH_DX + 1, TY = TH_DY + 1;
  __shared__ R s_f[4][PY * PX];
  __shared__ R s_ti[4][TY * TX], s_tj[4][TY * TX];
  const int G = cD.G, k = (int)blockIdx.x, l = (int)blockIdx.z;
  const int ntx = (G + TH_DX - 1) / TH_DX;
  const int i0 = ((int)blockIdx.y % ntx) * TH_DX, j0 = ((int)blockIdx.y / ntx) * TH_DY;
  const int tid = threadIdx.x;
  for (int p = tid; p < PX * PY; p += blockDim.x) {
    const int ii = i0 - 1 + p % PX, jj = j0 - 1 + p / PX;
    R f0 = R(0.0), f1 = R(0.0), f2 = R(0.0), f3 = R(0.0);
    if (ii >= 0 && jj >= 0 && ii < G && jj < G) {
      const int q = ix(ii, jj, k, l);
      const R rg = CG.RGAM[q];
      f0 = a.rho[q];
      f1 = a.rvx[q] * rg;
      f2 = a.rvy[q] * rg;
      f3 = a.rvz[q] * rg;
    }
    s_f[0][p] = f0; s_f[1][p] = f1; s_f[2][p] = f2; s_f[3][p] = f3;
  }
  __syncthreads();
  for (int p = tid; p < TX * TY; p += blockDim.x) {   // vertex values of (i0-1.., j0-1..)
    const int px = p % TX, py = p / TX;
    const int vi = i0 - 1 + px, vj = j0 - 1 + py;
    const bool ok = vi >= 0 && vj >= 0 && vi <= G - 2 && vj <= G - 2;
    R w1i = R(0.0), w2i = R(0.0), w3i = R(0.0), w1j = R(0.0), w2j = R(0.0), w3j = R(0.0);
    if (ok) {
      w1i = P2c(CG.GMTR_t, 0, vi, vj, l); w2i = P2c(CG.GMTR_t, 1, vi, vj, l); w3i = P2c(CG.GMTR_t, 2, vi, vj, l);
      w1j = P2c(CG.GMTR_t, 3, vi, vj, l); w2j = P2c(CG.GMTR_t, 4, vi, vj, l); w3j = P2c(CG.GMTR_t, 5, vi, vj, l);
    }
    const int ia = py * PX + px, ib = ia + 1, ic = ia + PX + 1, id = ia + PX;
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      R ti = R(0.0), tj = R(0.0);
      if (ok) {
        const R f0 = s_f[n][ia], fi = s_f[n][ib], fd = s_f[n][ic], fj = s_f[n][id];
        ti = f0 * w1i + fi * w2i;
        ti = ti + fd * w3i;
        tj = f0 * w1j;
        tj = tj + (fd * w2j + fj * w3j);
      }
      s_ti[n][p] = ti;
      s_tj[n][p] = tj;
    }
  }
  __syncthreads();
  if (i0 == 0 && j0 == 0 && tid < 4) {   // singular-point fix of vertex (0,0) (mod_src_tracer.py:1409-1412)
    const int v00 = 1 * TX + 1, v10 = 1 * TX + 2;
    const R m0 = (R)CG.pntmask[l * 2 + 0], m1 = (R)CG.pntmask[l * 2 + 1];
    s_ti[tid][v00] = s_ti[tid][v00] * m0 + s_tj[tid][v10] * m1;
  }
  __syncthreads();
  const int i = i0 + tid % TH_DX, j = j0 + tid / TH_DX;
  if (i >= G || j >= G) return;
  const int p = ix(i, j, k, l);
  const R dt = a.dt;
  const R PR = P2c(CG.GMTR_p, 0, i, j, l);
  const int vc = (j - j0 + 1) * TX + (i - i0 + 1);   // vertex (i, j); (i-1, j) is vc-1, (i, j-1) vc-TX
  // face f of the cell (ci, cj) from the vertex sums TA + TB (mod_src_tracer.py:1414-1484)
  auto face = [&](int ci, int cj, int f, int va, bool a_is_j, int vb, bool b_is_j, R xc[3]) {
    R sv[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      const R A = a_is_j ? s_tj[n][va] : s_ti[n][va];
      const R B = b_is_j ? s_tj[n][vb] : s_ti[n][vb];
      sv[n] = A + B;
    }
    return trc_face(a, ci, cj, l, f, sv, xc);
  };
  R fl[6], xc[3];
  // face 0: TJ(i, j-1) + TI(i, j)
  if (i >= 0 && i <= G - 2 && j >= 1 && j <= G - 2) {
    fl[0] = face(i, j, 0, vc - TX, true, vc, false, xc) * PR * dt;
  } else {
    fl[0] = R(0.0); xc[0] = xc[1] = xc[2] = R(0.0);
  }
  for (int d = 0; d < 3; ++d) a.xc[0 * 3 + d][p] = xc[d];
  // face 1: TI(i, j) + TJ(i, j)
  if (i >= 0 && i <= G - 2 && j >= 0 && j <= G - 2) {
    fl[1] = face(i, j, 1, vc, false, vc, true, xc) * PR * dt;
  } else {
    fl[1] = R(0.0); xc[0] = xc[1] = xc[2] = R(0.0);
  }
  for (int d = 0; d < 3; ++d) a.xc[1 * 3 + d][p] = xc[d];
  // face 2: TJ(i, j) + TI(i-1, j)
  if (i >= 1 && i <= G - 2 && j >= 0 && j <= G - 2) {
    fl[2] = face(i, j, 2, vc, true, vc - 1, false, xc) * PR * dt;
  } else {
    fl[2] = R(0.0); xc[0] = xc[1] = xc[2] = R(0.0);
  }
  for (int d = 0; d < 3; ++d) a.xc[2 * 3 + d][p] = xc[d];
  // faces 3..5: the neighbours' faces 0..2, opposite sign
  R xcn[3];
  fl[3] = (i - 1 >= 0 && i - 1 <= G - 2 && j >= 1 && j <= G - 2)
              ? -face(i - 1, j, 0, vc - 1 - TX, true, vc - 1, false, xcn) * PR * dt : R(0.0);
  fl[4] = (i - 1 >= 0 && i - 1 <= G - 2 && j - 1 >= 0 && j - 1 <= G - 2)
              ? -face(i - 1, j - 1, 1, vc - 1 - TX, false, vc - 1 - TX, true, xcn) * PR * dt : R(0.0);
  fl[5] = (i >= 1 && i <= G - 2 && j - 1 >= 0 && j - 1 <= G - 2)
              ? -face(i, j - 1, 2, vc - TX, true, vc - TX - 1, false, xcn) * PR * dt : R(0.0);
  if (i == 1 && j == 1) fl[5] *= (R)CG.pntmask[l * 2 + 0];
  const auto rg = recip_of(a.rhog_t[p]);   // six quotients by rhog_t
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    a.flx[f][p] = fl[f];
    const R chv = div_by(fl[f], rg);
    a.ch[f][p] = chv;
    a.cm[f][p] = R(0.5) - copysign(R(0.5), chv - CC.EPS);
  }
}

// pole edges (mod_src_tracer.py:1487-1531) and Courant numbers
template <class R>
struct TrcHfluxPlArgs {
  const R *rho, *rvx, *rvy, *rvz, *rhog_t;
  R *flx, *xc, *ch, *cm;   // flx/ch/cm (g,k,l); xc (g,k,l,3)
  R dt;
};

template <class R>
__global__ void k_trc_hflux_pl(TrcHfluxPlArgs<R> a) {
  int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  int k = t / cD.LP, lp = t % cD.LP;
  const R* gt = CG.GMTR_t_pl;
  const R* ga = CG.GMTR_a_pl;
  const R* gp = CG.GMTR_p_pl;
  R tv[6][4];
  auto F = [&](int n, int q) -> R {
    if (n == 0) return a.rho[q];
    const R* r = (n == 1) ? a.rvx : ((n == 2) ? a.rvy : a.rvz);
    return r[q] * gam_at(CG.RGAM_pl, q);
  };
  for (int v = 1; v <= 5; ++v) {
    int vp1 = (v + 1 == 6) ? 1 : v + 1;
    const R* g5 = gt + (v * cD.LP + lp) * 5;
    for (int n = 0; n < 4; ++n)
      tv[v][n] = F(n, ipl(0, k, lp)) * g5[2] + F(n, ipl(v, k, lp)) * g5[3] + F(n, ipl(vp1, k, lp)) * g5[4];
  }
  R rc = a.rhog_t[ipl(0, k, lp)];
  for (int v = 1; v <= 5; ++v) {
    int vm1 = (v - 1 == 0) ? 5 : v - 1;
    R rr2 = R(1.0) / npmax(tv[vm1][0] + tv[v][0], CC.EPS);
    R v2[3];
    for (int n = 0; n < 3; ++n) v2[n] = tv[vm1][n + 1] + tv[v][n + 1];
    const R* g18 = ga + (v * cD.LP + lp) * 18;
    R flux = R(0.5) * (v2[0] * g18[0] + v2[1] * g18[1] + v2[2] * g18[2]);
    int q = ipl(v, k, lp);
    R fl = flux * gp[(0 * cD.LP + lp) * 8 + 1] * a.dt;
    a.flx[q] = fl;
    for (int d = 0; d < 3; ++d) a.xc[q * 3 + d] = CG.GRD_xr_pl[(v * cD.LP + lp) * 3 + d] - v2[d] * rr2 * a.dt * R(0.5);
    R chv = fl / rc;
    a.ch[q] = chv;
    a.cm[q] = R(0.5) - copysign(R(0.5), chv - CC.EPS);
  }
}

// ---------------------------------------------------------------------------
// per tracer: q and its gradient (mod_src_tracer.py:758-771, 1634-1640)
// ---------------------------------------------------------------------------
// One block per (level, 32 x 8 tile of interior cells): q of the haloed tile
// is formed once into shared memory (one division per cell instead of one per
// stencil use), then each cell's gradient is read from there.  The region's
// halo cells get q and a zero gradient from the tile that holds their nearest
// interior cell, so every cell is written exactly once.
#define TG_DX 32
#define TG_DY 8
template <class R>
__global__ void __launch_bounds__(TG_DX * TG_DY) k_trc_grad_t(const R* rhogq, const R* rhog_t, R* q,
                                                              R* gq0, R* gq1, R* gq2) {
  constexpr int PX = TG_DX + 2, PY = TG_DY + 2;
  __shared__ R s_q[PY * PX];
  const TileLv tl = tile_level<TG_DX, TG_DY>(0);
  const int k = tl.k, l = tl.l, i0 = tl.i0, j0 = tl.j0;
  const int G = cD.G, gmax = cD.G - 2;
  const int tid = threadIdx.x;
  for (int p = tid; p < PX * PY; p += blockDim.x) {
    const int ii = i0 - 1 + p % PX, jj = j0 - 1 + p / PX;
    R v = R(0.0);
    if (ii < G && jj < G) {
      const int qq = ix(ii, jj, k, l);
      v = rhogq[qq] / rhog_t[qq];
      if (!interior(ii, jj)) {
        const int ci = min(max(ii, 1), gmax), cj = min(max(jj, 1), gmax);
        if (ci >= i0 && ci < i0 + TG_DX && cj >= j0 && cj < j0 + TG_DY) {
          q[qq] = v;
          gq0[qq] = R(0.0);
          gq1[qq] = R(0.0);
          gq2[qq] = R(0.0);
        }
      }
    }
    s_q[p] = v;
  }
  __syncthreads();
  const int tx = tid % TG_DX, ty = tid / TG_DX;
  const int i = i0 + tx, j = j0 + ty;
  if (i > gmax || j > gmax) return;
  const int qq = ix(i, j, k, l);
  const int c0 = (ty + 1) * PX + (tx + 1);
  const R s7[7] = {s_q[c0], s_q[c0 + 1], s_q[c0 + PX + 1], s_q[c0 + PX], s_q[c0 - 1], s_q[c0 - PX - 1], s_q[c0 - PX]};
  q[qq] = s7[0];
  R* gq[3] = {gq0, gq1, gq2};
#pragma unroll
  for (int d = 0; d < 3; ++d) {   // grad7 (kernels/oprtgradient.py:45-70)
    R a = P2c(CG.coef_grad, d * 7 + 0, i, j, l) * s7[0];
#pragma unroll
    for (int m = 1; m < 7; ++m) a = a + P2c(CG.coef_grad, d * 7 + m, i, j, l) * s7[m];
    gq[d][qq] = a;
  }
}

template <class R>
__global__ void k_trc_grad_pl(const R* rhogq, const R* rhog_t, R* q, R* gq0, R* gq1,
                              R* gq2) {
  int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  int k = t / cD.LP, lp = t % cD.LP;
  R qv[6];
  for (int v = 0; v < 6; ++v) {
    int p = ipl(v, k, lp);
    qv[v] = rhogq[p] / rhog_t[p];
    q[p] = qv[v];
  }
  R* gq[3] = {gq0, gq1, gq2};
  for (int d = 0; d < 3; ++d) {
    R row = R(0.0);
    for (int v = 0; v < 6; ++v) {
      R tv = CG.coef_grad_pl[(v * cD.LP + lp) * 3 + d] * qv[v];
      row = (v == 0) ? tv : row + tv;
    }
    gq[d][ipl(0, k, lp)] = row;
    for (int v = 1; v < 6; ++v) gq[d][ipl(v, k, lp)] = R(0.0);
  }
}

// ---------------------------------------------------------------------------
// MIURA2004 face values of edges 0..2 (mod_src_tracer.py:1696-1787)
// ---------------------------------------------------------------------------
template <class R>
struct TrcRemapArgs {
  const R *q, *gq0, *gq1, *gq2;
  const R* xc[9];
  const R* cm[6];
  R* qa[3];
};

template <class R>
__device__ __forceinline__ R trc_rec(const TrcRemapArgs<R>& a, int ii, int jj, int k, int l, int pxc, int f) {
  int q = ix(ii, jj, k, l);
  R r = a.q[q];
  r = r + a.gq0[q] * (a.xc[f * 3 + 0][pxc] - P2(CG.GRD_x, 0, ii, jj, l));
  r = r + a.gq1[q] * (a.xc[f * 3 + 1][pxc] - P2(CG.GRD_x, 1, ii, jj, l));
  r = r + a.gq2[q] * (a.xc[f * 3 + 2][pxc] - P2(CG.GRD_x, 2, ii, jj, l));
  return r;
}

template <class R>
__global__ void k_trc_remap(TrcRemapArgs<R> a) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l;
  if (!col_of(t, i, j, l)) return;
  const int G = cD.G;
  const bool ok = (i <= G - 2 && j <= G - 2);
  for (int k = 0; k < cD.KA; ++k) {
    int p = ix(i, j, k, l);
    if (!ok) {
      a.qa[0][p] = R(0.0); a.qa[1][p] = R(0.0); a.qa[2][p] = R(0.0);
      continue;
    }
    const int mi[3] = {1, 1, 0}, mj[3] = {0, 1, 1};
    for (int f = 0; f < 3; ++f) {
      R ap = trc_rec(a, i, j, k, l, p, f);
      R am = trc_rec(a, i + mi[f], j + mj[f], k, l, p, f);
      R c = a.cm[f][p];
      a.qa[f][p] = c * am + (R(1.0) - c) * ap;
    }
  }
}

template <class R>
struct TrcRemapPlArgs {
  const R *q, *gq0, *gq1, *gq2, *xc, *cm;
  R* qa;
};

template <class R>
__global__ void k_trc_remap_pl(TrcRemapPlArgs<R> a) {
  int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  int k = t / cD.LP, lp = t % cD.LP;
  const R* X = CG.GRD_x_pl;
  const R* gq[3] = {a.gq0, a.gq1, a.gq2};
  int p0 = ipl(0, k, lp);
  for (int v = 1; v <= 5; ++v) {
    int pv = ipl(v, k, lp);
    R ap = a.q[p0];
    for (int d = 0; d < 3; ++d) ap = ap + gq[d][p0] * (a.xc[pv * 3 + d] - X[(0 * cD.LP + lp) * 3 + d]);
    R am = a.q[pv];
    for (int d = 0; d < 3; ++d) am = am + gq[d][pv] * (a.xc[pv * 3 + d] - X[(v * cD.LP + lp) * 3 + d]);
    R c = a.cm[pv];
    a.qa[pv] = c * am + (R(1.0) - c) * ap;
  }
}

// ---------------------------------------------------------------------------
// horizontal Thuburn limiter (mod_src_tracer.py:2190-2605, numpy branch)
// ---------------------------------------------------------------------------
template <class R>
struct TrcLimArgs {
  const R *q, *rhog_t, *frhog;
  const R* ch[6];
  const R* cm[6];
  const R* qa[3];
  const R *qout_min, *qout_max;
  R *Qmin, *Qmax;          // Qout (output of the Qout kernel)
  const R* flx[6];
  R* rhogq;
  R dt;
};

// q_min / q_max over the stencil of edge f of cell (a,b) (mod_src_tracer.py:2191-2217)
template <class R>
__device__ void trc_face_minmax(const R* q, int a, int b, int k, int l, int f, R& qn, R& qx) {
  auto Q = [&](int ii, int jj) { return q[ix(ii, jj, k, l)]; };
  R q0 = Q(a, b);
  R q2 = Q(a + 1, b), q3 = Q(a + 1, b + 1), qj = Q(a, b + 1);
  R v1, v2, v3;
  if (f == 0) {
    R q1 = (b > 0) ? Q(a, b - 1) : Q(0, 0);
    v1 = q1; v2 = q2; v3 = q3;
  } else if (f == 1) {
    v1 = q2; v2 = q3; v3 = qj;
  } else {
    R q4 = (a > 0) ? Q(a - 1, b) : Q(0, 0);
    v1 = q3; v2 = qj; v3 = q4;
  }
  qn = npmin(npmin(npmin(q0, v1), v2), v3);
  qx = npmax(npmax(npmax(q0, v1), v2), v3);
}

// Qin of slot m (0..5) of cell (i,j): slots 0..2 from the cell's own edges,
// slots 3..5 from the neighbours' edges 0..2 (mod_src_tracer.py:2220-2234 and
// the singular-point override :2298-2323)
template <class R>
__device__ void trc_qin(const TrcLimArgs<R>& a, int i, int j, int k, int l, int m, R& qin_min, R& qin_max) {
  const R BIG = CC.HUGE_;
  int ai = i, bj = j, f = m;
  if (m >= 3) {
    const int nbI[3] = {-1, -1, 0}, nbJ[3] = {0, -1, -1};
    ai = i + nbI[m - 3];
    bj = j + nbJ[m - 3];
    f = m - 3;
  }
  R cmv = a.cm[f][ix(ai, bj, k, l)];
  R qn, qx;
  const bool sgp = CG.have_sgp[l] && ai == 0 && bj == 0 && f == 1;
  if (sgp) {
    auto Q = [&](int ii, int jj) { return a.q[ix(ii, jj, k, l)]; };
    // np.min over [q(0,0), q(1,1), q(2,1), q(0,1)]
    qn = npmin(npmin(npmin(Q(0, 0), Q(1, 1)), Q(2, 1)), Q(0, 1));
    qx = npmax(npmax(npmax(Q(0, 0), Q(1, 1)), Q(2, 1)), Q(0, 1));
    if (m < 3) {
      qin_min = (cmv == R(1.0)) ? qn : BIG;
      qin_max = (cmv == R(1.0)) ? qx : -BIG;
    } else {
      qin_min = (cmv == R(1.0)) ? BIG : qn;
      qin_max = (cmv == R(1.0)) ? -BIG : qx;
    }
    return;
  }
  trc_face_minmax(a.q, ai, bj, k, l, f, qn, qx);
  if (m < 3) {
    qin_min = cmv * qn + (R(1.0) - cmv) * BIG;
    qin_max = cmv * qx + (R(1.0) - cmv) * (-BIG);
  } else {
    qin_min = cmv * BIG + (R(1.0) - cmv) * qn;
    qin_max = cmv * (-BIG) + (R(1.0) - cmv) * qx;
  }
}

template <class R>
__global__ void k_trc_qout(TrcLimArgs<R> a) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l;
  if (!col_of(t, i, j, l)) return;
  const bool in = interior(i, j);
  const R EPS = CC.EPS;
  for (int k = 0; k < cD.KA; ++k) {
    int p = ix(i, j, k, l);
    R qc = a.q[p];
    if (!in) {
      a.Qmin[p] = qc;
      a.Qmax[p] = qc;
      continue;
    }
    R qnmin = qc, qnmax = qc;
    R Cin = R(0.0), Cout = R(0.0), CQmin = R(0.0), CQmax = R(0.0);
    for (int m = 0; m < 6; ++m) {
      R qi, qx;
      trc_qin(a, i, j, k, l, m, qi, qx);
      qnmin = npmin(qnmin, qi);
      qnmax = npmax(qnmax, qx);
      R chv = a.ch[m][p];
      R chm = npmin(chv, R(0.0));
      if (m == 0) {
        Cin = chm; Cout = chv - chm; CQmin = chm * qi; CQmax = chm * qx;
      } else {
        Cin = Cin + chm; Cout = Cout + (chv - chm); CQmin = CQmin + chm * qi; CQmax = CQmax + chm * qx;
      }
    }
    R zsw = R(0.5) - copysign(R(0.5), fabs(Cout) - EPS);
    R d = R(1.0) * a.frhog[p] / a.rhog_t[p] * a.dt;
    a.Qmin[p] = (qc - CQmax - qnmax * (R(1.0) - Cin - Cout + d)) / (Cout + zsw) * (R(1.0) - zsw) + qc * zsw;
    a.Qmax[p] = (qc - CQmin - qnmin * (R(1.0) - Cin - Cout + d)) / (Cout + zsw) * (R(1.0) - zsw) + qc * zsw;
  }
}

// limited value of edge f in {0,1,2} of cell (ai,bj) (mod_src_tracer.py:2545-2605)
template <class R>
__device__ R trc_limited_face(const TrcLimArgs<R>& a, int ai, int bj, int k, int l, int f) {
  const int mi[3] = {1, 1, 0}, mj[3] = {0, 1, 1};
  int ni = ai + mi[f], nj = bj + mj[f];
  int p = ix(ai, bj, k, l), pn = ix(ni, nj, k, l);
  R c = a.cm[f][p];
  R qa = a.qa[f][p];
  R qi0, qx0, qi1, qx1;
  trc_qin(a, ai, bj, k, l, f, qi0, qx0);
  trc_qin(a, ni, nj, k, l, 3 + f, qi1, qx1);
  qa = c * npmin(npmax(qa, qi0), qx0) + (R(1.0) - c) * npmin(npmax(qa, qi1), qx1);
  qa = c * npmax(npmin(qa, a.qout_max[pn]), a.qout_min[pn]) + (R(1.0) - c) * npmax(npmin(qa, a.qout_max[p]), a.qout_min[p]);
  return qa;
}

template <class R>
__global__ void k_trc_apply(TrcLimArgs<R> a) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l;
  if (!col_of(t, i, j, l)) return;
  if (!interior(i, j)) return;
  for (int k = 0; k < cD.KA; ++k) {
    int p = ix(i, j, k, l);
    R q0 = trc_limited_face(a, i, j, k, l, 0);
    R q1 = trc_limited_face(a, i, j, k, l, 1);
    R q2 = trc_limited_face(a, i, j, k, l, 2);
    R q3 = trc_limited_face(a, i - 1, j, k, l, 0);
    R q4 = trc_limited_face(a, i - 1, j - 1, k, l, 1);
    R q5 = trc_limited_face(a, i, j - 1, k, l, 2);
    R upd = a.flx[0][p] * q0 + a.flx[1][p] * q1 + a.flx[2][p] * q2 + a.flx[3][p] * q3 + a.flx[4][p] * q4 +
                 a.flx[5][p] * q5;
    a.rhogq[p] = a.rhogq[p] - upd;
  }
}

// pole Qout (mod_src_tracer.py:2437-2495) at g = 0
template <class R>
struct TrcLimPlArgs {
  const R *q, *ch, *cm, *rhog_t, *frhog, *qa, *flx;
  R *Qmin, *Qmax;
  const R *qout_min, *qout_max;
  R* rhogq;
  R dt;
};

template <class R>
__device__ void trc_qin_pl(const TrcLimPlArgs<R>& a, int v, int k, int lp, R& in0n, R& in1n, R& in0x,
                           R& in1x) {
  const R BIG = CC.HUGE_;
  int vp1 = (v + 1 > 5) ? 1 : v + 1, vm1 = (v - 1 < 1) ? 5 : v - 1;
  R q0 = a.q[ipl(0, k, lp)], qv = a.q[ipl(v, k, lp)], qm = a.q[ipl(vm1, k, lp)], qp = a.q[ipl(vp1, k, lp)];
  R qn = pymin(pymin(pymin(q0, qv), qm), qp);
  R qx = pymax(pymax(pymax(q0, qv), qm), qp);
  R c = a.cm[ipl(v, k, lp)];
  in0n = (c == R(1.0)) ? qn : BIG;
  in1n = (c == R(1.0)) ? BIG : qn;
  in0x = (c == R(1.0)) ? qx : -BIG;
  in1x = (c == R(1.0)) ? -BIG : qx;
}

template <class R>
__global__ void k_trc_qout_pl(TrcLimPlArgs<R> a) {
  int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  int k = t / cD.LP, lp = t % cD.LP;
  int p0 = ipl(0, k, lp);
  R qnm = a.q[p0], qnx = a.q[p0];
  R in0n[6], in0x[6], d1, d2;
  for (int v = 1; v <= 5; ++v) {
    trc_qin_pl(a, v, k, lp, in0n[v], d1, in0x[v], d2);
    qnm = pymin(qnm, in0n[v]);
    qnx = pymax(qnx, in0x[v]);
  }
  R Ci = R(0.0), Co = R(0.0), CQn = R(0.0), CQx = R(0.0);
  for (int v = 1; v <= 5; ++v) {
    int pv = ipl(v, k, lp);
    R chm = a.cm[pv] * a.ch[pv];
    Ci = Ci + chm;
    Co = Co + (a.ch[pv] - chm);
    CQn = CQn + chm * in0n[v];
    CQx = CQx + chm * in0x[v];
  }
  R zs = R(0.5) - copysign(R(0.5), fabs(Co) - CC.EPS);
  R den = Co + zs;
  R fac = R(1.0) - zs;
  R q0 = a.q[p0];
  R dv = R(1.0) * a.frhog[p0] / a.rhog_t[p0] * a.dt;
  a.Qmin[p0] = (q0 - CQx - qnx * (R(1.0) - Ci - Co + dv)) / den * fac + q0 * zs;
  a.Qmax[p0] = (q0 - CQn - qnm * (R(1.0) - Ci - Co + dv)) / den * fac + q0 * zs;
}

template <class R>
__global__ void k_trc_apply_pl(TrcLimPlArgs<R> a) {
  int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  int k = t / cD.LP, lp = t % cD.LP;
  int p0 = ipl(0, k, lp);
  R acc = a.rhogq[p0];
  for (int v = 1; v <= 5; ++v) {
    int pv = ipl(v, k, lp);
    R in0n, in1n, in0x, in1x;
    trc_qin_pl(a, v, k, lp, in0n, in1n, in0x, in1x);
    R c = a.cm[pv];
    R x = a.qa[pv];
    R a0 = npmin(npmax(x, in0n), in0x);
    R a1 = npmin(npmax(x, in1n), in1x);
    x = c * a0 + (R(1.0) - c) * a1;
    R a2 = npmax(npmin(x, a.qout_max[pv]), a.qout_min[pv]);
    R a3 = npmax(npmin(x, a.qout_max[p0]), a.qout_min[p0]);
    x = c * a2 + (R(1.0) - c) * a3;
    acc = acc - a.flx[pv] * x;
  }
  a.rhogq[p0] = acc;
}

// density after the horizontal step (mod_src_tracer.py:890-916)
template <class R>
__global__ void k_trc_rhog(R* rhog_t, const R* f0, const R* f1, const R* f2, const R* f3,
                           const R* f4, const R* f5, const R* frhog, R dt, const R* flx_pl,
                           R* rhog_t_pl, const R* frhog_pl) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l;
  if (col_of(t, i, j, l)) {
    if (!interior(i, j)) return;
    for (int k = 0; k < cD.KA; ++k) {
      int p = ix(i, j, k, l);
      R s = f0[p] + f1[p] + f2[p] + f3[p] + f4[p] + f5[p];
      rhog_t[p] = rhog_t[p] - (s - (R(1.0) * frhog[p] * dt));
    }
  } else {
    int tp = t - cD.npt2i;
    if (tp < cD.KA * cD.LP) {
      int k = (int)(tp / cD.LP), lp = (int)(tp % cD.LP);
      int p0 = ipl(0, k, lp);
      R r = rhog_t_pl[p0];
      for (int v = 1; v <= 5; ++v) r = r - flx_pl[ipl(v, k, lp)];
      r = r + R(1.0) * frhog_pl[p0] * dt;
      rhog_t_pl[p0] = r;
    }
  }
}

}  // namespace nc
