// Tangent-linear and adjoint kernels of step operators (float64), for the
// differentiable path behind torch.autograd.Function (adjoint.py):
//
// * the HEVI vertical implicit solve (kernels/virhowsolver.py:67-122): per
//   column the tridiagonal system Ml x[n-1] + Mc x[n] + Mu x[n+1] = b[n] on the
//   levels kmin+1..kmax, solved by the Thomas algorithm; its adjoint is the
//   solve with the transposed matrix (sub-diagonal Mu[n-1], super-diagonal
//   Ml[n+1]);
// * one vertical tracer advection step with the vertical Thuburn limiter
//   (mod_src_tracer.py:389-533, 1909-2074; the forward arithmetic is that of
//   trc_vadv_column): the tangent-linear and adjoint of the step at a given
//   tracer state, with the limiter's branches (upwind side, min / max
//   choices, the final clamp of tiny negatives) those of the forward
//   evaluation -- the active-branch linearisation; the density, fluxes and
//   Courant numbers are fixed inputs;
// * the horizontal Laplacian (kernels/oprtlaplacian.py:41-55, the pole row
//   :143-157) after the halo exchange: y = L(C(q)) on interior cells and the
//   pole points; the adjoint C^T L^T, with the exchange's adjoint adding each
//   halo value back into its source cell.
#pragma once
#include "nc_tracer.cuh"

namespace nc {

// levels held per thread by the column kernels below (local arrays); the
// entry points refuse grids with more
#define NC_ADJ_K 64

// ---------------------------------------------------------------------------
// tridiagonal solve and its transpose, one thread per regional column
// ---------------------------------------------------------------------------
struct TriArgs {
  const double *Mc, *Mu, *Ml, *b;
  double* x;
  // with the transposed solve: the forward solution and the cotangents of the
  // matrix entries (-lambda[n] x[n], -lambda[n] x[n+1], -lambda[n] x[n-1]),
  // written when x_fwd is not null
  const double* x_fwd;
  double *gMc, *gMu, *gMl;
  int transpose;
};

__device__ void tri_column(const Col c, const TriArgs& a) {
  const int k0 = cD.kmin + 1, N = cD.kmax - cD.kmin, KA = cD.KA;
  // row n: lo(n) x[n-1] + Mc[n] x[n] + up(n) x[n+1] = b[n]
  auto lo = [&](int n) { return a.transpose ? a.Mu[c.at(k0 + n - 1)] : a.Ml[c.at(k0 + n)]; };
  auto up = [&](int n) { return a.transpose ? a.Ml[c.at(k0 + n + 1)] : a.Mu[c.at(k0 + n)]; };
  double u[NC_ADJ_K], gam[NC_ADJ_K];
  double beta = a.Mc[c.at(k0)];
  u[0] = a.b[c.at(k0)] / beta;
  for (int n = 1; n < N; ++n) {
    gam[n] = up(n - 1) / beta;
    beta = a.Mc[c.at(k0 + n)] - lo(n) * gam[n];
    u[n] = (a.b[c.at(k0 + n)] - lo(n) * u[n - 1]) / beta;
  }
  for (int n = N - 2; n >= 0; --n) u[n] = u[n] - gam[n + 1] * u[n + 1];
  for (int k = 0; k < KA; ++k) a.x[c.at(k)] = (k >= k0 && k < k0 + N) ? u[k - k0] : 0.0;
  if (!a.x_fwd) return;
  for (int k = 0; k < KA; ++k) {
    const int n = k - k0;
    double gc = 0.0, gu = 0.0, gl = 0.0;
    if (n >= 0 && n < N) {
      gc = -u[n] * a.x_fwd[c.at(k)];
      if (n + 1 < N) gu = -u[n] * a.x_fwd[c.at(k + 1)];
      if (n > 0) gl = -u[n] * a.x_fwd[c.at(k - 1)];
    }
    a.gMc[c.at(k)] = gc;
    a.gMu[c.at(k)] = gu;
    a.gMl[c.at(k)] = gl;
  }
}

__global__ void k_tri_solve(TriArgs a, int pole) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  int i, j, l, g, lp;
  if (!map_col(pole, t, i, j, l, g, lp)) return;
  tri_column(pole ? col_pl(g, lp) : col_reg(i, j, l), a);
}

// ---------------------------------------------------------------------------
// vertical tracer advection step: forward, tangent-linear, adjoint
// ---------------------------------------------------------------------------
struct VadvLin {
  const double *rhogq, *den, *flx_v, *frhog;   // linearisation point and the fixed inputs
  const double* in;                            // TL: perturbation of rhogq; AD: adjoint of the output
  double* out;                                 // forward: F(rhogq); TL: perturbation of F; AD: adjoint of rhogq
  double dt, bcoef;
  int clamp, mode;                             // mode 0 forward, 1 tangent-linear, 2 adjoint
};

// the argument npmin / npmax return (0 the first, 1 the second; on ties the
// second, as they do): the linearisation follows the forward's choice
__device__ __forceinline__ int amin2(double a, double b) { return (a < b) ? 0 : 1; }
__device__ __forceinline__ int amax2(double a, double b) { return (a > b) ? 0 : 1; }

__device__ void vadv_lin_column(const Col c, const VadvLin& a) {
  const int KA = cD.KA, kmin = cD.kmin, kmax = cD.kmax;
  const double BIG = cC.HUGE_, EPS = cC.EPS;
  double q[NC_ADJ_K], raw[NC_ADJ_K], omin[NC_ADJ_K], omax[NC_ADJ_K];
  double fk[NC_ADJ_K], zk[NC_ADJ_K], Ak[NC_ADJ_K], c1v[NC_ADJ_K], c2v[NC_ADJ_K];
  // branch record per level: upwind sides; argument of the Q bounds (0 qc, 1 neighbour);
  // qnmin / qnmax (0 QL, 1 QU, 2 qc); limited face (0 raw, 1 lower bound, 2 upper bound)
  signed char inL[NC_ADJ_K], inU[NC_ADJ_K], sminL[NC_ADJ_K], sminU[NC_ADJ_K], smaxL[NC_ADJ_K], smaxU[NC_ADJ_K];
  signed char snmin[NC_ADJ_K], snmax[NC_ADJ_K], sh[NC_ADJ_K];
  bool clamped[NC_ADJ_K];
  for (int k = 0; k < KA; ++k) q[k] = a.rhogq[c.at(k)] / a.den[c.at(k)];
  for (int k = kmin; k <= kmax + 1; ++k) raw[k] = cC.afact[k] * q[k] + cC.bfact[k] * q[k - 1];
  for (int k = kmin; k <= kmax; ++k) {
    const int p = c.at(k);
    const double denk = a.den[p];
    const double ck0 = -a.flx_v[p] / denk * cC.rdgz[k];
    const double ck1 = a.flx_v[c.at(k + 1)] / denk * cC.rdgz[k];
    const double ck0p = (k + 1 <= kmax) ? -a.flx_v[c.at(k + 1)] / a.den[c.at(k + 1)] * cC.rdgz[k + 1] : 0.0;
    const double L = 0.5 - copysign(0.5, ck0), U = 0.5 + copysign(0.5, ck0p);
    inL[k] = (L == 1.0);
    inU[k] = (U == 1.0);
    const double qc = q[k], qb = q[k - 1], qa = q[k + 1];
    sminL[k] = amin2(qc, qb); smaxL[k] = amax2(qc, qb);
    sminU[k] = amin2(qc, qa); smaxU[k] = amax2(qc, qa);
    const double QminL = inL[k] ? (sminL[k] ? qb : qc) : BIG, QmaxL = inL[k] ? (smaxL[k] ? qb : qc) : -BIG;
    const double QminU = inU[k] ? (sminU[k] ? qa : qc) : BIG, QmaxU = inU[k] ? (smaxU[k] ? qa : qc) : -BIG;
    const int s1 = amin2(QminL, QminU);
    const double m1 = s1 ? QminU : QminL;
    snmin[k] = amin2(m1, qc) ? 2 : s1;
    const double qnmin = (snmin[k] == 2) ? qc : m1;
    const int s2 = amax2(QmaxL, QmaxU);
    const double x1 = s2 ? QmaxU : QmaxL;
    snmax[k] = amax2(x1, qc) ? 2 : s2;
    const double qnmax = (snmax[k] == 2) ? qc : x1;
    const double Cin = L * ck0 + U * ck1, Cout = (1.0 - L) * ck0 + (1.0 - U) * ck1;
    const double CQmin = L * ck0 * QminL + U * ck1 * QminU, CQmax = L * ck0 * QmaxL + U * ck1 * QmaxU;
    const double zsw = 0.5 - copysign(0.5, fabs(Cout) - EPS);
    const double dk = a.bcoef * a.frhog[p] / denk * a.dt;
    const double A = Cin + Cout - dk;
    omin[k] = ((qc - qnmax) + qnmax * A - CQmax) / (Cout + zsw) * (1.0 - zsw) + qc * zsw;
    omax[k] = ((qc - qnmin) + qnmin * A - CQmin) / (Cout + zsw) * (1.0 - zsw) + qc * zsw;
    fk[k] = (1.0 - zsw) / (Cout + zsw);
    zk[k] = zsw;
    Ak[k] = A;
    c1v[k] = L * ck0;
    c2v[k] = U * ck1;
  }
  // limited faces qh[k] on k = kmin+1..kmax, zero at kmin and kmax+1: the
  // bounds of the upwind cell, k-1 when inflow comes from below (inL)
  double qh[NC_ADJ_K];
  for (int k = 0; k < KA; ++k) qh[k] = 0.0;
  for (int k = kmin + 1; k <= kmax; ++k) {
    const int jb = inL[k] ? k - 1 : k;
    const double lo = omin[jb], hi = omax[jb];
    const int s_lo = amax2(raw[k], lo);            // np.maximum(raw, lo)
    const double mx = s_lo ? lo : raw[k];
    const int s_hi = amin2(mx, hi);                // np.minimum(mx, hi)
    sh[k] = s_hi ? 2 : (s_lo ? 1 : 0);
    qh[k] = s_hi ? hi : mx;
  }
  for (int k = 0; k < KA; ++k) clamped[k] = false;
  if (a.mode == 0) {
    for (int k = 0; k < KA; ++k) a.out[c.at(k)] = 0.0;
    for (int k = kmin; k <= kmax; ++k) {
      double x = a.rhogq[c.at(k)] - (a.flx_v[c.at(k + 1)] * qh[k + 1] - a.flx_v[c.at(k)] * qh[k]) * cC.rdgz[k];
      if (a.clamp && x > -1.0e-10 && x < 0.0) x = 0.0;
      a.out[c.at(k)] = x;
    }
    return;
  }
  for (int k = kmin; k <= kmax; ++k) {
    const double x = a.rhogq[c.at(k)] - (a.flx_v[c.at(k + 1)] * qh[k + 1] - a.flx_v[c.at(k)] * qh[k]) * cC.rdgz[k];
    clamped[k] = a.clamp && x > -1.0e-10 && x < 0.0;
  }
  if (a.mode == 1) {
    // tangent-linear: the same sequence on perturbations
    double dq[NC_ADJ_K], draw[NC_ADJ_K], dmin[NC_ADJ_K], dmax[NC_ADJ_K], dqh[NC_ADJ_K];
    for (int k = 0; k < KA; ++k) {
      dq[k] = a.in[c.at(k)] / a.den[c.at(k)];
      dqh[k] = 0.0;
    }
    for (int k = kmin; k <= kmax + 1; ++k) draw[k] = cC.afact[k] * dq[k] + cC.bfact[k] * dq[k - 1];
    for (int k = kmin; k <= kmax; ++k) {
      const double dc = dq[k];
      const double dminL = inL[k] ? (sminL[k] ? dq[k - 1] : dc) : 0.0, dmaxL = inL[k] ? (smaxL[k] ? dq[k - 1] : dc) : 0.0;
      const double dminU = inU[k] ? (sminU[k] ? dq[k + 1] : dc) : 0.0, dmaxU = inU[k] ? (smaxU[k] ? dq[k + 1] : dc) : 0.0;
      const double dnmin = (snmin[k] == 2) ? dc : (snmin[k] == 1 ? dminU : dminL);
      const double dnmax = (snmax[k] == 2) ? dc : (snmax[k] == 1 ? dmaxU : dmaxL);
      const double dCQmin = c1v[k] * dminL + c2v[k] * dminU, dCQmax = c1v[k] * dmaxL + c2v[k] * dmaxU;
      // qomin = f (qc - qnmax + A qnmax - CQmax) + zsw qc
      dmin[k] = fk[k] * (dc + (Ak[k] - 1.0) * dnmax - dCQmax) + zk[k] * dc;
      dmax[k] = fk[k] * (dc + (Ak[k] - 1.0) * dnmin - dCQmin) + zk[k] * dc;
    }
    for (int k = kmin + 1; k <= kmax; ++k) {
      const int jb = inL[k] ? k - 1 : k;
      dqh[k] = (sh[k] == 0) ? draw[k] : (sh[k] == 1 ? dmin[jb] : dmax[jb]);
    }
    for (int k = 0; k < KA; ++k) a.out[c.at(k)] = 0.0;
    for (int k = kmin; k <= kmax; ++k) {
      const double d = a.in[c.at(k)] - (a.flx_v[c.at(k + 1)] * dqh[k + 1] - a.flx_v[c.at(k)] * dqh[k]) * cC.rdgz[k];
      a.out[c.at(k)] = clamped[k] ? 0.0 : d;
    }
    return;
  }
  // adjoint: the tangent-linear steps transposed, in reverse order
  double gy[NC_ADJ_K], gqh[NC_ADJ_K], graw[NC_ADJ_K], gmin[NC_ADJ_K], gmax[NC_ADJ_K], gq[NC_ADJ_K], gr[NC_ADJ_K];
  for (int k = 0; k < KA; ++k) {
    gy[k] = (k >= kmin && k <= kmax && !clamped[k]) ? a.in[c.at(k)] : 0.0;
    gqh[k] = graw[k] = gmin[k] = gmax[k] = gq[k] = gr[k] = 0.0;
  }
  for (int k = kmin; k <= kmax; ++k) {   // out_k = in_k - (flx_{k+1} qh_{k+1} - flx_k qh_k) rdgz_k
    gr[k] += gy[k];
    gqh[k + 1] -= a.flx_v[c.at(k + 1)] * cC.rdgz[k] * gy[k];
    gqh[k] += a.flx_v[c.at(k)] * cC.rdgz[k] * gy[k];
  }
  for (int k = kmin + 1; k <= kmax; ++k) {
    const int jb = inL[k] ? k - 1 : k;
    if (sh[k] == 0) graw[k] += gqh[k];
    else if (sh[k] == 1) gmin[jb] += gqh[k];
    else gmax[jb] += gqh[k];
  }
  for (int k = kmin; k <= kmax; ++k) {
    // dmin = (f + zsw) dc + f (A - 1) dnmax - f dCQmax, and the same for dmax with qnmin / CQmin
    gq[k] += (fk[k] + zk[k]) * (gmin[k] + gmax[k]);
    const double gnmax = fk[k] * (Ak[k] - 1.0) * gmin[k], gCQmax = -fk[k] * gmin[k];
    const double gnmin = fk[k] * (Ak[k] - 1.0) * gmax[k], gCQmin = -fk[k] * gmax[k];
    double gminL = c1v[k] * gCQmin, gminU = c2v[k] * gCQmin, gmaxL = c1v[k] * gCQmax, gmaxU = c2v[k] * gCQmax;
    if (snmin[k] == 2) gq[k] += gnmin;
    else if (snmin[k] == 1) gminU += gnmin;
    else gminL += gnmin;
    if (snmax[k] == 2) gq[k] += gnmax;
    else if (snmax[k] == 1) gmaxU += gnmax;
    else gmaxL += gnmax;
    if (inL[k]) {
      gq[sminL[k] ? k - 1 : k] += gminL;
      gq[smaxL[k] ? k - 1 : k] += gmaxL;
    }
    if (inU[k]) {
      gq[sminU[k] ? k + 1 : k] += gminU;
      gq[smaxU[k] ? k + 1 : k] += gmaxU;
    }
  }
  for (int k = kmin; k <= kmax + 1; ++k) {   // raw_k = afact_k q_k + bfact_k q_{k-1}
    gq[k] += cC.afact[k] * graw[k];
    gq[k - 1] += cC.bfact[k] * graw[k];
  }
  for (int k = 0; k < KA; ++k) a.out[c.at(k)] = gr[k] + gq[k] / a.den[c.at(k)];
}

__global__ void k_vadv_lin(VadvLin a, int pole) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  int i, j, l, g, lp;
  if (!map_col(pole, t, i, j, l, g, lp)) return;
  vadv_lin_column(pole ? col_pl(g, lp) : col_reg(i, j, l), a);
}

// ---------------------------------------------------------------------------
// horizontal Laplacian and its adjoint (the exchange first / its adjoint last)
// ---------------------------------------------------------------------------
// y = L(q) on interior cells (halo cells 0); pole point row g = 0, neighbours 0
__global__ void k_lap_fwd(const double* q, double* y) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.npti) return;
  const int G = cD.G, KA = cD.KA;
  const int i = t % G, j = (t / G) % G, k = (t / (G * G)) % KA, l = t / (G * G * KA);
  double v = 0.0;
  if (interior(i, j)) v = lap7<double>(i, j, k, l, [&](int ii, int jj, int kk) { return q[ix(ii, jj, kk, l)]; });
  y[t] = v;
}
__global__ void k_lap_fwd_pl(const double* q, double* y) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP;
  double row = 0.0;
  for (int v = 0; v < 6; ++v) {
    const double tv = cG.coef_lap_pl[v * cD.LP + lp] * q[ipl(v, k, lp)];
    row = (v == 0) ? tv : row + tv;
  }
  y[ipl(0, k, lp)] = row;
  for (int g = 1; g < 6; ++g) y[ipl(g, k, lp)] = 0.0;
}
// the transposed stencil: every cell gathers coef_lap[m](i) y(i) from the
// interior cells i whose stencil point m it is
__global__ void k_lap_adj(const double* y, double* g) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.npti) return;
  const int G = cD.G, KA = cD.KA;
  const int i = t % G, j = (t / G) % G, k = (t / (G * G)) % KA, l = t / (G * G * KA);
  double s = 0.0;
  for (int m = 0; m < 7; ++m) {
    const int si = i - kNbI[m], sj = j - kNbJ[m];
    if (si >= 0 && sj >= 0 && si < G && sj < G && interior(si, sj))
      s += P2(cG.coef_lap, m, si, sj, l) * y[ix(si, sj, k, l)];
  }
  g[t] = s;
}
__global__ void k_lap_adj_pl(const double* y, double* g) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP;
  const double y0 = y[ipl(0, k, lp)];
  for (int v = 0; v < 6; ++v) g[ipl(v, k, lp)] = cG.coef_lap_pl[v * cD.LP + lp] * y0;
}
// adjoint of the halo exchange on one field: each destination's value is added
// to its source (atomically: several destinations may share a source), then
// the destinations are cleared by k_comm_adj_clear
__global__ void k_comm_adj_add(double* r, double* p, const long long* r_dst, const long long* r_src, int nr,
                               const long long* p_dst, const long long* p_src, int np) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nent = nr + np;
  if (t >= (long long)nent * cD.KA) return;
  const int k = (int)(t / nent), e = (int)(t % nent);
  const long long pl = cD.plane;
  auto reg_at = [&](long long cidx) { return ((cidx / pl) * cD.KA + k) * pl + cidx % pl; };
  if (e < nr) {
    const double v = r[reg_at(r_dst[e])];
    const long long s = r_src[e];
    if (s >= 0) atomicAdd(&r[reg_at(s)], v);
    else {
      const long long gp = -s - 1;
      atomicAdd(&p[ipl((int)(gp / cD.LP), k, (int)(gp % cD.LP))], v);
    }
  } else {
    const int ee = e - nr;
    const long long gp = p_dst[ee];
    const double v = p[ipl((int)(gp / cD.LP), k, (int)(gp % cD.LP))];
    atomicAdd(&r[reg_at(p_src[ee])], v);
  }
}
__global__ void k_comm_adj_clear(double* r, double* p, const long long* r_dst, int nr, const long long* p_dst,
                                 int np) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nent = nr + np;
  if (t >= (long long)nent * cD.KA) return;
  const int k = (int)(t / nent), e = (int)(t % nent);
  const long long pl = cD.plane;
  if (e < nr) {
    const long long d = r_dst[e];
    r[((d / pl) * cD.KA + k) * pl + d % pl] = 0.0;
  } else {
    const long long gp = p_dst[e - nr];
    p[ipl((int)(gp / cD.LP), k, (int)(gp % cD.LP))] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// horizontal tracer step (mod_src_tracer.py:758-916, 1634-1787, 2190-2605):
// tangent-linear and adjoint at a forward evaluation.  The forward arrays q,
// qa (face values), Qmin / Qmax (after their exchange) of that evaluation are
// given; every min / max of the limiter is re-decided from them exactly as
// the forward kernels decide it, and the linearised value follows the chosen
// argument (a constant +-HUGE contributes nothing).
// ---------------------------------------------------------------------------
enum { SRC_NONE = 0, SRC_Q = 1, SRC_QA = 2, SRC_QMIN = 3, SRC_QMAX = 4 };
struct Src {
  int kind, idx, f;   // f: face of a SRC_QA source
};

struct HLin {
  // forward evaluation
  const double *q, *qa[3], *Qmin, *Qmax, *rhog_t, *frhog;
  const double *ch[6], *cm[6], *flx[6], *xc[9];
  // pole arrays: q, qa, Qmin / Qmax (g, k, lp); ch / cm / flx (g, k, lp); xc (g, k, lp, 3)
  const double *q_pl, *qa_pl, *Qmin_pl, *Qmax_pl, *rhog_t_pl, *frhog_pl, *ch_pl, *cm_pl, *flx_pl, *xc_pl;
  double dt;
  // tangent-linear: inputs dq, dqa, dQmin / dQmax; outputs dQmin / dQmax (qout) or y (apply)
  // adjoint: cotangents accumulated into gq, gqa, gQmin / gQmax
  const double *dq, *dqa[3], *dQmin, *dQmax, *dq_pl, *dqa_pl, *dQmin_pl, *dQmax_pl;
  double *oQmin, *oQmax, *oQmin_pl, *oQmax_pl;
  const double *x, *x_pl;   // apply: the step's input perturbation (TL) / output cotangent (AD)
  double *y, *y_pl;         // apply TL output
  double *gq, *gqa[3], *gQmin, *gQmax, *gq_pl, *gqa_pl, *gQmin_pl, *gQmax_pl;
  double *gg[3], *gg_pl[3];   // cotangents of the (exchanged) gradient
  double *gx, *gx_pl;         // cotangent of the step's input, accumulated
};

// indices of the min / max over the stencil of edge f of cell (a, b)
// (trc_face_minmax: npmin / npmax chains in the same order)
__device__ void face_minmax_idx(const double* q, int a, int b, int k, int l, int f, int& imin, int& imax) {
  auto I = [&](int ii, int jj) { return ix(ii, jj, k, l); };
  const int i0 = I(a, b), i2 = I(a + 1, b), i3 = I(a + 1, b + 1), ij = I(a, b + 1);
  int v[3];
  if (f == 0) {
    v[0] = (b > 0) ? I(a, b - 1) : I(0, 0); v[1] = i2; v[2] = i3;
  } else if (f == 1) {
    v[0] = i2; v[1] = i3; v[2] = ij;
  } else {
    v[0] = i3; v[1] = ij; v[2] = (a > 0) ? I(a - 1, b) : I(0, 0);
  }
  int m = i0, M = i0;
  for (int n = 0; n < 3; ++n) {
    if (!(q[m] < q[v[n]])) m = v[n];
    if (!(q[M] > q[v[n]])) M = v[n];
  }
  imin = m;
  imax = M;
}

// Qin of slot m of cell (i, j) (trc_qin): value and source of the min / max
__device__ void qin_src(const HLin& a, int i, int j, int k, int l, int m, double& vmin, double& vmax, Src& smin,
                        Src& smax) {
  const double BIG = cC.HUGE_;
  int ai = i, bj = j, f = m;
  if (m >= 3) {
    const int nbI[3] = {-1, -1, 0}, nbJ[3] = {0, -1, -1};
    ai = i + nbI[m - 3];
    bj = j + nbJ[m - 3];
    f = m - 3;
  }
  const double cmv = a.cm[f][ix(ai, bj, k, l)];
  int imin, imax;
  if (cG.have_sgp[l] && ai == 0 && bj == 0 && f == 1) {
    const int c4[4] = {ix(0, 0, k, l), ix(1, 1, k, l), ix(2, 1, k, l), ix(0, 1, k, l)};
    imin = imax = c4[0];
    for (int n = 1; n < 4; ++n) {
      if (!(a.q[imin] < a.q[c4[n]])) imin = c4[n];
      if (!(a.q[imax] > a.q[c4[n]])) imax = c4[n];
    }
  } else {
    face_minmax_idx(a.q, ai, bj, k, l, f, imin, imax);
  }
  const bool use = (m < 3) ? (cmv == 1.0) : (cmv != 1.0);
  if (use) {
    vmin = a.q[imin]; vmax = a.q[imax];
    smin = Src{SRC_Q, imin, 0}; smax = Src{SRC_Q, imax, 0};
  } else {
    vmin = BIG; vmax = -BIG;
    smin = Src{SRC_NONE, 0, 0}; smax = Src{SRC_NONE, 0, 0};
  }
}

// npmin(npmax(x, lo), hi) and npmax(npmin(x, hi), lo) with their sources
__device__ __forceinline__ void clamp_minmax(double& x, Src& sx, double lo, Src slo, double hi, Src shi) {
  if (!(x > lo)) { x = lo; sx = slo; }
  if (!(x < hi)) { x = hi; sx = shi; }
}
__device__ __forceinline__ void clamp_maxmin(double& x, Src& sx, double lo, Src slo, double hi, Src shi) {
  if (!(x < hi)) { x = hi; sx = shi; }
  if (!(x > lo)) { x = lo; sx = slo; }
}

// source of the limited value of edge f of cell (ai, bj) (trc_limited_face)
__device__ Src limited_face_src(const HLin& a, int ai, int bj, int k, int l, int f) {
  const int mi[3] = {1, 1, 0}, mj[3] = {0, 1, 1};
  const int ni = ai + mi[f], nj = bj + mj[f];
  const int p = ix(ai, bj, k, l), pn = ix(ni, nj, k, l);
  const bool c = a.cm[f][p] == 1.0;
  double v = a.qa[f][p];
  Src sv{SRC_QA, p, f};
  double lo, hi;
  Src slo, shi;
  if (c) qin_src(a, ai, bj, k, l, f, lo, hi, slo, shi);
  else qin_src(a, ni, nj, k, l, 3 + f, lo, hi, slo, shi);
  clamp_minmax(v, sv, lo, slo, hi, shi);
  const int pc = c ? pn : p;
  clamp_maxmin(v, sv, a.Qmin[pc], Src{SRC_QMIN, pc, 0}, a.Qmax[pc], Src{SRC_QMAX, pc, 0});
  return sv;
}

__device__ __forceinline__ double src_tl(const HLin& a, Src s) {
  switch (s.kind) {
    case SRC_Q: return a.dq[s.idx];
    case SRC_QA: return a.dqa[s.f][s.idx];
    case SRC_QMIN: return a.dQmin[s.idx];
    case SRC_QMAX: return a.dQmax[s.idx];
    default: return 0.0;
  }
}
__device__ __forceinline__ void src_ad(const HLin& a, Src s, double v) {
  switch (s.kind) {
    case SRC_Q: atomicAdd(&a.gq[s.idx], v); break;
    case SRC_QA: atomicAdd(&a.gqa[s.f][s.idx], v); break;
    case SRC_QMIN: atomicAdd(&a.gQmin[s.idx], v); break;
    case SRC_QMAX: atomicAdd(&a.gQmax[s.idx], v); break;
    default: break;
  }
}

// Qout of an interior cell as a linear form of q at the forward's branches
// (k_trc_qout): Qmin = fz qc + sum wmin_n q[smin_n], the same for Qmax
struct QoutLin {
  double fz, B, f;
  Src nmin, nmax, imin[6], imax[6];
  double chm[6];
};
__device__ void qout_lin(const HLin& a, int i, int j, int k, int l, QoutLin& o) {
  const int p = ix(i, j, k, l);
  const double qc = a.q[p];
  double qnmin = qc, qnmax = qc, Cin = 0.0, Cout = 0.0;
  o.nmin = o.nmax = Src{SRC_Q, p, 0};
  for (int m = 0; m < 6; ++m) {
    double qi, qx;
    qin_src(a, i, j, k, l, m, qi, qx, o.imin[m], o.imax[m]);
    if (!(qnmin < qi)) { qnmin = qi; o.nmin = o.imin[m]; }
    if (!(qnmax > qx)) { qnmax = qx; o.nmax = o.imax[m]; }
    const double chv = a.ch[m][p];
    const double chm = (chv < 0.0) ? chv : 0.0;
    o.chm[m] = chm;
    if (m == 0) { Cin = chm; Cout = chv - chm; }
    else { Cin = Cin + chm; Cout = Cout + (chv - chm); }
  }
  const double zsw = 0.5 - copysign(0.5, fabs(Cout) - cC.EPS);
  const double d = 1.0 * a.frhog[p] / a.rhog_t[p] * a.dt;
  o.B = 1.0 - Cin - Cout + d;
  o.f = (1.0 - zsw) / (Cout + zsw);
  o.fz = o.f + zsw;
}

__global__ void k_hlin_qout(HLin a, int adjoint) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  int i, j, l;
  if (!col_of(t, i, j, l)) return;
  const bool in = interior(i, j);
  for (int k = 0; k < cD.KA; ++k) {
    const int p = ix(i, j, k, l);
    if (!in) {   // Qmin = Qmax = q
      if (adjoint) atomicAdd(&a.gq[p], a.gQmin[p] + a.gQmax[p]);
      else { a.oQmin[p] = a.dq[p]; a.oQmax[p] = a.dq[p]; }
      continue;
    }
    QoutLin o;
    qout_lin(a, i, j, k, l, o);
    if (!adjoint) {
      double cqmin = 0.0, cqmax = 0.0;
      for (int m = 0; m < 6; ++m) {
        cqmin += o.chm[m] * src_tl(a, o.imin[m]);
        cqmax += o.chm[m] * src_tl(a, o.imax[m]);
      }
      a.oQmin[p] = o.fz * a.dq[p] - o.f * cqmax - o.f * o.B * src_tl(a, o.nmax);
      a.oQmax[p] = o.fz * a.dq[p] - o.f * cqmin - o.f * o.B * src_tl(a, o.nmin);
    } else {
      const double gn = a.gQmin[p], gx = a.gQmax[p];
      atomicAdd(&a.gq[p], o.fz * (gn + gx));
      for (int m = 0; m < 6; ++m) {
        src_ad(a, o.imax[m], -o.f * o.chm[m] * gn);
        src_ad(a, o.imin[m], -o.f * o.chm[m] * gx);
      }
      src_ad(a, o.nmax, -o.f * o.B * gn);
      src_ad(a, o.nmin, -o.f * o.B * gx);
    }
  }
}

// the flux update of the interior cells (k_trc_apply): y = x - sum flx_f v_f
__global__ void k_hlin_apply(HLin a, int adjoint) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  int i, j, l;
  if (!col_of(t, i, j, l)) return;
  const bool in = interior(i, j);
  for (int k = 0; k < cD.KA; ++k) {
    const int p = ix(i, j, k, l);
    if (!in) {
      if (!adjoint) a.y[p] = a.x[p];
      continue;
    }
    const Src s[6] = {limited_face_src(a, i, j, k, l, 0),     limited_face_src(a, i, j, k, l, 1),
                      limited_face_src(a, i, j, k, l, 2),     limited_face_src(a, i - 1, j, k, l, 0),
                      limited_face_src(a, i - 1, j - 1, k, l, 1), limited_face_src(a, i, j - 1, k, l, 2)};
    if (!adjoint) {
      double upd = 0.0;
      for (int f = 0; f < 6; ++f) upd += a.flx[f][p] * src_tl(a, s[f]);
      a.y[p] = a.x[p] - upd;
    } else {
      const double g = a.x[p];
      for (int f = 0; f < 6; ++f) src_ad(a, s[f], -a.flx[f][p] * g);
    }
  }
}

// MIURA2004 face values (k_trc_remap), adjoint: scatter into gq and the gradient cotangents
__global__ void k_hlin_remap_ad(HLin a) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  int i, j, l;
  if (!col_of(t, i, j, l)) return;
  const int G = cD.G;
  if (i > G - 2 || j > G - 2) return;
  const int mi[3] = {1, 1, 0}, mj[3] = {0, 1, 1};
  for (int k = 0; k < cD.KA; ++k) {
    const int p = ix(i, j, k, l);
    for (int f = 0; f < 3; ++f) {
      const double g = a.gqa[f][p];
      if (g == 0.0) continue;
      const double c = a.cm[f][p];
      const int ni = i + mi[f], nj = j + mj[f], pn = ix(ni, nj, k, l);
      atomicAdd(&a.gq[p], (1.0 - c) * g);
      atomicAdd(&a.gq[pn], c * g);
      for (int d = 0; d < 3; ++d) {
        const double xcv = a.xc[f * 3 + d][p];
        atomicAdd(&a.gg[d][p], (1.0 - c) * g * (xcv - P2(cG.GRD_x, d, i, j, l)));
        atomicAdd(&a.gg[d][pn], c * g * (xcv - P2(cG.GRD_x, d, ni, nj, l)));
      }
    }
  }
}

// gradient (k_trc_grad_t) adjoint on the interior cells, then x-bar +=
// q-bar / rhog_t on every regional cell
__global__ void k_hlin_grad_ad(HLin a) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.npti) return;
  const int G = cD.G, KA = cD.KA;
  const int i = t % G, j = (t / G) % G, k = (t / (G * G)) % KA, l = t / (G * G * KA);
  double s = 0.0;
  for (int m = 0; m < 7; ++m) {   // every interior cell whose stencil point m is (i, j)
    const int si = i - kNbI[m], sj = j - kNbJ[m];
    if (si >= 1 && sj >= 1 && si <= G - 2 && sj <= G - 2) {
      const int ps = ix(si, sj, k, l);
      for (int d = 0; d < 3; ++d) s += P2(cG.coef_grad, d * 7 + m, si, sj, l) * a.gg[d][ps];
    }
  }
  a.gx[t] += (a.gq[t] + s) / a.rhog_t[t];
}

// ---- pole point (g = 0) of each pole and level
__device__ void qin_pl_src(const HLin& a, int v, int k, int lp, double& in0n, double& in1n, double& in0x,
                           double& in1x, Src& sn, Src& sx, bool& c1) {
  const double BIG = cC.HUGE_;
  const int vp1 = (v + 1 > 5) ? 1 : v + 1, vm1 = (v - 1 < 1) ? 5 : v - 1;
  const int c4[4] = {ipl(0, k, lp), ipl(v, k, lp), ipl(vm1, k, lp), ipl(vp1, k, lp)};
  int imin = c4[0], imax = c4[0];
  for (int n = 1; n < 4; ++n) {   // pymin / pymax: the later argument only when strictly beyond
    if (a.q_pl[c4[n]] < a.q_pl[imin]) imin = c4[n];
    if (a.q_pl[c4[n]] > a.q_pl[imax]) imax = c4[n];
  }
  c1 = a.cm_pl[ipl(v, k, lp)] == 1.0;
  const double qn = a.q_pl[imin], qx = a.q_pl[imax];
  in0n = c1 ? qn : BIG;
  in1n = c1 ? BIG : qn;
  in0x = c1 ? qx : -BIG;
  in1x = c1 ? -BIG : qx;
  sn = Src{SRC_Q, imin, 0};
  sx = Src{SRC_Q, imax, 0};
}

__device__ __forceinline__ double src_tl_pl(const HLin& a, Src s) {
  switch (s.kind) {
    case SRC_Q: return a.dq_pl[s.idx];
    case SRC_QA: return a.dqa_pl[s.idx];
    case SRC_QMIN: return a.dQmin_pl[s.idx];
    case SRC_QMAX: return a.dQmax_pl[s.idx];
    default: return 0.0;
  }
}
__device__ __forceinline__ void src_ad_pl(const HLin& a, Src s, double v) {
  switch (s.kind) {
    case SRC_Q: atomicAdd(&a.gq_pl[s.idx], v); break;
    case SRC_QA: atomicAdd(&a.gqa_pl[s.idx], v); break;
    case SRC_QMIN: atomicAdd(&a.gQmin_pl[s.idx], v); break;
    case SRC_QMAX: atomicAdd(&a.gQmax_pl[s.idx], v); break;
    default: break;
  }
}

// pole Qout (k_trc_qout_pl) and flux update (k_trc_apply_pl): one thread per (k, lp)
__global__ void k_hlin_pole(HLin a, int adjoint, int stage) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP;
  const int p0 = ipl(0, k, lp);
  if (stage == 0) {   // Qout at p0
    double qnm = a.q_pl[p0], qnx = a.q_pl[p0];
    Src snm{SRC_Q, p0, 0}, snx{SRC_Q, p0, 0}, sn[6], sx[6];
    double chm[6], Ci = 0.0, Co = 0.0;
    for (int v = 1; v <= 5; ++v) {
      double in0n, in1n, in0x, in1x;
      bool c1;
      qin_pl_src(a, v, k, lp, in0n, in1n, in0x, in1x, sn[v], sx[v], c1);
      if (!c1) sn[v] = sx[v] = Src{SRC_NONE, 0, 0};
      if (in0n < qnm) { qnm = in0n; snm = sn[v]; }
      if (in0x > qnx) { qnx = in0x; snx = sx[v]; }
      const int pv = ipl(v, k, lp);
      chm[v] = a.cm_pl[pv] * a.ch_pl[pv];
      Ci = Ci + chm[v];
      Co = Co + (a.ch_pl[pv] - chm[v]);
    }
    const double zs = 0.5 - copysign(0.5, fabs(Co) - cC.EPS);
    const double f = (1.0 - zs) / (Co + zs), fz = f + zs;
    const double B = 1.0 - Ci - Co + 1.0 * a.frhog_pl[p0] / a.rhog_t_pl[p0] * a.dt;
    if (!adjoint) {
      double cqn = 0.0, cqx = 0.0;
      for (int v = 1; v <= 5; ++v) {
        cqn += chm[v] * src_tl_pl(a, sn[v]);
        cqx += chm[v] * src_tl_pl(a, sx[v]);
      }
      a.oQmin_pl[p0] = fz * a.dq_pl[p0] - f * cqx - f * B * src_tl_pl(a, snx);
      a.oQmax_pl[p0] = fz * a.dq_pl[p0] - f * cqn - f * B * src_tl_pl(a, snm);
    } else {
      const double gn = a.gQmin_pl[p0], gx = a.gQmax_pl[p0];
      atomicAdd(&a.gq_pl[p0], fz * (gn + gx));
      for (int v = 1; v <= 5; ++v) {
        src_ad_pl(a, sx[v], -f * chm[v] * gn);
        src_ad_pl(a, sn[v], -f * chm[v] * gx);
      }
      src_ad_pl(a, snx, -f * B * gn);
      src_ad_pl(a, snm, -f * B * gx);
    }
    return;
  }
  // stage 1: flux update of p0 from its five edges (the other pole points keep x)
  double acc = 0.0;
  const double g = adjoint ? a.x_pl[p0] : 0.0;
  for (int v = 1; v <= 5; ++v) {
    const int pv = ipl(v, k, lp);
    double in0n, in1n, in0x, in1x;
    Src sn, sx;
    bool c1;
    qin_pl_src(a, v, k, lp, in0n, in1n, in0x, in1x, sn, sx, c1);
    const Src none{SRC_NONE, 0, 0};
    double x = a.qa_pl[pv];
    Src s{SRC_QA, pv, 0};
    if (c1) clamp_minmax(x, s, in0n, sn, in0x, sx);        // a0, chosen by c = 1
    else clamp_minmax(x, s, in1n, sn, in1x, sx);           // a1
    (void)none;
    const int pc = c1 ? pv : p0;
    clamp_maxmin(x, s, a.Qmin_pl[pc], Src{SRC_QMIN, pc, 0}, a.Qmax_pl[pc], Src{SRC_QMAX, pc, 0});
    if (!adjoint) acc += a.flx_pl[pv] * src_tl_pl(a, s);
    else src_ad_pl(a, s, -a.flx_pl[pv] * g);
  }
  if (!adjoint) {
    for (int v = 0; v < 6; ++v) a.y_pl[ipl(v, k, lp)] = a.x_pl[ipl(v, k, lp)];
    a.y_pl[p0] = a.x_pl[p0] - acc;
  }
}

// pole remap (k_trc_remap_pl) adjoint: one thread per (k, lp); before the
// gradient cotangents' exchange adjoint
__global__ void k_hlin_pole_remap_ad(HLin a) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP;
  const int p0 = ipl(0, k, lp);
  const double* X = cG.GRD_x_pl;
  // qa[pv] = c am + (1 - c) ap, ap from p0, am from pv
  for (int v = 1; v <= 5; ++v) {
    const int pv = ipl(v, k, lp);
    const double g = a.gqa_pl[pv], c = a.cm_pl[pv];
    a.gq_pl[p0] += (1.0 - c) * g;
    a.gq_pl[pv] += c * g;
    for (int d = 0; d < 3; ++d) {
      a.gg_pl[d][p0] += (1.0 - c) * g * (a.xc_pl[pv * 3 + d] - X[(0 * cD.LP + lp) * 3 + d]);
      a.gg_pl[d][pv] += c * g * (a.xc_pl[pv * 3 + d] - X[(v * cD.LP + lp) * 3 + d]);
    }
  }
}

// pole gradient (k_trc_grad_pl) adjoint, then x-bar += q-bar / rhog_t on the
// pole arrays: gq_d[p0] = sum_v coef_grad_pl(v, d) q[v], the other rows zero
__global__ void k_hlin_pole_grad_ad(HLin a) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP;
  const int p0 = ipl(0, k, lp);
  for (int d = 0; d < 3; ++d) {
    const double g = a.gg_pl[d][p0];
    for (int v = 0; v < 6; ++v) a.gq_pl[ipl(v, k, lp)] += cG.coef_grad_pl[(v * cD.LP + lp) * 3 + d] * g;
  }
  for (int v = 0; v < 6; ++v) {
    const int pv = ipl(v, k, lp);
    a.gx_pl[pv] += a.gq_pl[pv] / a.rhog_t_pl[pv];
  }
}

// ---------------------------------------------------------------------------
// divergence (kernels/fluxconv.py:52-108) and gradient
// (kernels/oprtgradient.py:45-88) after the halo exchange, and their
// adjoints.  Three-component fields are stored one component after the other
// (3 x npt regional, 3 x npl pole values).
// ---------------------------------------------------------------------------
__global__ void k_div_fwd(const double* v, double* y) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.npti) return;
  const int G = cD.G, KA = cD.KA, n = cD.npti;
  const int i = t % G, j = (t / G) % G, k = (t / (G * G)) % KA, l = t / (G * G * KA);
  double r = 0.0;
  if (interior(i, j))
    r = div7<double>(i, j, k, l, [&](int ii, int jj, int kk, int d) { return v[d * n + ix(ii, jj, kk, l)]; });
  y[t] = r;
}
__global__ void k_div_fwd_pl(const double* v, double* y) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP, np = cD.npl;
  double row = 0.0;
  for (int g = 0; g < 6; ++g) {
    const int q = ipl(g, k, lp);
    const double* cd = cG.coef_div_pl + (g * cD.LP + lp) * 3;
    const double pv = cd[0] * v[q] + cd[1] * v[np + q] + cd[2] * v[2 * np + q];
    row = (g == 0) ? pv : row + pv;
  }
  y[ipl(0, k, lp)] = row;
  for (int g = 1; g < 6; ++g) y[ipl(g, k, lp)] = 0.0;
}
// v-bar_d at every cell: the interior cells s whose stencil point m it is
__global__ void k_div_adj(const double* y, double* v) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.npti) return;
  const int G = cD.G, KA = cD.KA, n = cD.npti;
  const int i = t % G, j = (t / G) % G, k = (t / (G * G)) % KA, l = t / (G * G * KA);
  double acc[3] = {0.0, 0.0, 0.0};
  for (int m = 0; m < 7; ++m) {
    const int si = i - kNbI[m], sj = j - kNbJ[m];
    if (si >= 1 && sj >= 1 && si <= G - 2 && sj <= G - 2) {
      const double ys = y[ix(si, sj, k, l)];
      for (int d = 0; d < 3; ++d) acc[d] += P2(cG.coef_div, d * 7 + m, si, sj, l) * ys;
    }
  }
  for (int d = 0; d < 3; ++d) v[d * n + t] = acc[d];
}
__global__ void k_div_adj_pl(const double* y, double* v) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP, np = cD.npl;
  const double y0 = y[ipl(0, k, lp)];
  for (int g = 0; g < 6; ++g) {
    const int q = ipl(g, k, lp);
    const double* cd = cG.coef_div_pl + (g * cD.LP + lp) * 3;
    for (int d = 0; d < 3; ++d) v[d * np + q] = cd[d] * y0;
  }
}
__global__ void k_grad_fwd(const double* q, double* gr) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.npti) return;
  const int G = cD.G, KA = cD.KA, n = cD.npti;
  const int i = t % G, j = (t / G) % G, k = (t / (G * G)) % KA, l = t / (G * G * KA);
  double o[3] = {0.0, 0.0, 0.0};
  if (interior(i, j)) grad7<double>(i, j, k, l, [&](int ii, int jj, int kk) { return q[ix(ii, jj, kk, l)]; }, o);
  for (int d = 0; d < 3; ++d) gr[d * n + t] = o[d];
}
__global__ void k_grad_fwd_pl(const double* q, double* gr) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP, np = cD.npl;
  for (int d = 0; d < 3; ++d) {
    double row = 0.0;
    for (int g = 0; g < 6; ++g) {
      const double tv = cG.coef_grad_pl[(g * cD.LP + lp) * 3 + d] * q[ipl(g, k, lp)];
      row = (g == 0) ? tv : row + tv;
    }
    gr[d * np + ipl(0, k, lp)] = row;
    for (int g = 1; g < 6; ++g) gr[d * np + ipl(g, k, lp)] = 0.0;
  }
}
__global__ void k_grad_adj(const double* gr, double* q) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.npti) return;
  const int G = cD.G, KA = cD.KA, n = cD.npti;
  const int i = t % G, j = (t / G) % G, k = (t / (G * G)) % KA, l = t / (G * G * KA);
  double acc = 0.0;
  for (int m = 0; m < 7; ++m) {
    const int si = i - kNbI[m], sj = j - kNbJ[m];
    if (si >= 1 && sj >= 1 && si <= G - 2 && sj <= G - 2) {
      const int ps = ix(si, sj, k, l);
      for (int d = 0; d < 3; ++d) acc += P2(cG.coef_grad, d * 7 + m, si, sj, l) * gr[d * n + ps];
    }
  }
  q[t] = acc;
}
__global__ void k_grad_adj_pl(const double* gr, double* q) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP, np = cD.npl;
  const int p0 = ipl(0, k, lp);
  for (int g = 0; g < 6; ++g) {
    double acc = 0.0;
    for (int d = 0; d < 3; ++d) acc += cG.coef_grad_pl[(g * cD.LP + lp) * 3 + d] * gr[d * np + p0];
    q[ipl(g, k, lp)] = acc;
  }
}

// ---------------------------------------------------------------------------
// Kh-weighted horizontal diffusion (kernels/oprtdiffusion.py, the scalar pass
// of the hyperdiffusion: OPRT_diffusion of s with the coefficient field kh)
// after the halo exchange, and its adjoint.  y = D(C(s)) on interior cells and
// the pole point; linear in s for a given kh.  The triangle values of the
// forward are
//   TI(i,j) = (wI1 s(i,j) + wI2 s(i+1,j) + wI3 s(i+1,j+1)) / 3,
//   TJ(i,j) = (wJ1 s(i,j) + wJ2 s(i+1,j+1) + wJ3 s(i,j+1)) / 3
// per direction d (weights intp_w), with the singular-point fix at (0,0),
// TI(0,0) <- TI(0,0) m0 + TJ(1,0) m1; the cell sums the six edge terms
// kf_e cd_e (T + T') (kf_e the mean of kh at the cell and its e-th
// neighbour).  The adjoint gathers, for every triangle, the edge weights of
// the (up to three) cells that use it, undoes the fix, then gathers for
// every point the weights of the triangles that hold it.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool tri_ok(int ii, int jj) { return ii >= 0 && jj >= 0 && ii <= cD.G - 2 && jj <= cD.G - 2; }

// raw triangle value (before the singular-point fix), direction d, t = 0: TI, 1: TJ
__device__ __forceinline__ double diff_tri(const double* s, int ii, int jj, int k, int l, int d, int t) {
  if (!tri_ok(ii, jj)) return 0.0;
  const double w1 = P2(cG.intp_w, (d * 3 + 0) * 2 + t, ii, jj, l);
  const double w2 = P2(cG.intp_w, (d * 3 + 1) * 2 + t, ii, jj, l);
  const double w3 = P2(cG.intp_w, (d * 3 + 2) * 2 + t, ii, jj, l);
  const double s0 = s[ix(ii, jj, k, l)], sd = s[ix(ii + 1, jj + 1, k, l)];
  return t == 0 ? div3(w1 * s0 + w2 * s[ix(ii + 1, jj, k, l)] + w3 * sd)
                : div3(w1 * s0 + w2 * sd + w3 * s[ix(ii, jj + 1, k, l)]);
}
__device__ __forceinline__ double diff_tri_fixed(const double* s, int ii, int jj, int k, int l, int d, int t) {
  double v = diff_tri(s, ii, jj, k, l, d, t);
  if (t == 0 && ii == 0 && jj == 0)
    v = v * (double)cG.pntmask[l * 2 + 0] + diff_tri(s, 1, 0, k, l, d, 1) * (double)cG.pntmask[l * 2 + 1];
  return v;
}
// the six edge weights kf_e (e = 1..6 at index e - 1) of interior cell (i, j)
__device__ __forceinline__ void diff_kf(const double* kh, int i, int j, int k, int l, double kf[6]) {
  const double k0 = kh[ix(i, j, k, l)];
  kf[0] = 0.5 * (k0 + kh[ix(i + 1, j + 1, k, l)]);
  kf[1] = 0.5 * (k0 + kh[ix(i, j + 1, k, l)]);
  kf[2] = 0.5 * (k0 + kh[ix(i - 1, j, k, l)]);
  kf[3] = 0.5 * (k0 + kh[ix(i - 1, j - 1, k, l)]);
  kf[4] = 0.5 * (k0 + kh[ix(i, j - 1, k, l)]);
  kf[5] = 0.5 * (k0 + kh[ix(i + 1, j, k, l)]);
}

__global__ void k_diff_fwd(const double* kh, const double* s, double* y) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.npti) return;
  const int G = cD.G, KA = cD.KA;
  const int i = t % G, j = (t / G) % G, k = (t / (G * G)) % KA, l = t / (G * G * KA);
  double inner = 0.0;
  if (interior(i, j)) {
    double kf[6];
    diff_kf(kh, i, j, k, l, kf);
    for (int d = 0; d < 3; ++d) {
      const double aTI = diff_tri_fixed(s, i, j, k, l, d, 0), aTJ = diff_tri_fixed(s, i, j, k, l, d, 1);
      const double bTI = diff_tri_fixed(s, i - 1, j, k, l, d, 0);
      const double cTI = diff_tri_fixed(s, i - 1, j - 1, k, l, d, 0), cTJ = diff_tri_fixed(s, i - 1, j - 1, k, l, d, 1);
      const double dTJ = diff_tri_fixed(s, i, j - 1, k, l, d, 1);
      auto cd = [&](int e) { return P2(cG.coef_diff, d * 6 + e, i, j, l); };
      const double blk = kf[0] * cd(0) * (aTI + aTJ) + kf[1] * cd(1) * (aTJ + bTI) + kf[2] * cd(2) * (bTI + cTJ) +
                         kf[3] * cd(3) * (cTJ + cTI) + kf[4] * cd(4) * (cTI + dTJ) + kf[5] * cd(5) * (dTJ + aTI);
      inner = (d == 0) ? blk : inner + blk;
    }
  }
  y[t] = inner;
}

// the pole row (kernels/oprtdiffusion.py:137-177): the pole point from the
// five ring triangles; the ring rows are zero
__global__ void k_diff_fwd_pl(const double* kh, const double* s, double* y) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP;
  const double sn = s[ipl(0, k, lp)];
  double vt[5][3];
  for (int v = 1; v <= 5; ++v) {
    const int vp1 = (v == 5) ? 1 : v + 1;
    const double sij = s[ipl(v, k, lp)], sp1 = s[ipl(vp1, k, lp)];
    for (int d = 0; d < 3; ++d) {
      const double* cI = cG.coef_intp_pl + ((v * cD.LP + lp) * 3 + d) * 3;
      const double c0 = cI[0], c1 = cI[1], c2 = cI[2];
      vt[v - 1][d] = div3((2.0 * c0 - c1 - c2) * sn + (-c0 + 2.0 * c1 - c2) * sij + (-c0 - c1 + 2.0 * c2) * sp1);
    }
  }
  const double khn = kh[ipl(0, k, lp)];
  double row = 0.0;
  for (int v = 1; v <= 5; ++v) {
    const int vm1 = (v == 1) ? 5 : v - 1;
    const double kavg = 0.5 * (khn + kh[ipl(v, k, lp)]);
    double sd = 0.0;
    for (int d = 0; d < 3; ++d) {
      const double tv = cG.coef_diff_pl[(v * cD.LP + lp) * 3 + d] * (vt[vm1 - 1][d] + vt[v - 1][d]);
      sd = (d == 0) ? tv : sd + tv;
    }
    const double contrib = kavg * sd;
    row = (v == 1) ? contrib : row + contrib;
  }
  y[ipl(0, k, lp)] = row;
  for (int g = 1; g < 6; ++g) y[ipl(g, k, lp)] = 0.0;
}

// cotangent of the raw (unfixed) triangle value from the cells that use it
__device__ double diff_tbar_gathered(const double* kh, const double* y, int ii, int jj, int k, int l, int d, int t) {
  double acc = 0.0;
  double kf[6];
  auto cd = [&](int e, int ci, int cj) { return P2(cG.coef_diff, d * 6 + e, ci, cj, l); };
  // TI(ii,jj): cell (ii,jj) edges 1, 6; cell (ii+1,jj) edges 2, 3; cell (ii+1,jj+1) edges 4, 5
  // TJ(ii,jj): cell (ii,jj) edges 1, 2; cell (ii+1,jj+1) edges 3, 4; cell (ii,jj+1) edges 5, 6
  const int ci[3] = {ii, ii + 1, t == 0 ? ii + 1 : ii};
  const int cj[3] = {jj, t == 0 ? jj : jj + 1, jj + 1};
  const int e0[3] = {0, t == 0 ? 1 : 2, t == 0 ? 3 : 4};
  const int e1[3] = {t == 0 ? 5 : 1, t == 0 ? 2 : 3, t == 0 ? 4 : 5};
  for (int c = 0; c < 3; ++c) {
    const int i = ci[c], j = cj[c];
    if (i < 1 || j < 1 || i > cD.G - 2 || j > cD.G - 2) continue;
    diff_kf(kh, i, j, k, l, kf);
    acc += y[ix(i, j, k, l)] * (kf[e0[c]] * cd(e0[c], i, j) + kf[e1[c]] * cd(e1[c], i, j));
  }
  return acc;
}

// per triangle point: the cotangents of its two raw triangle values, three
// directions each (tb[(t * 3 + d) * npt + point]), the singular-point fix undone
__global__ void k_diff_adj_tri(const double* kh, const double* y, double* tb) {
  const int p = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (p >= cD.npti) return;
  const int G = cD.G, KA = cD.KA, n = cD.npti;
  const int ii = p % G, jj = (p / G) % G, k = (p / (G * G)) % KA, l = p / (G * G * KA);
  for (int t = 0; t < 2; ++t)
    for (int d = 0; d < 3; ++d) {
      double v = 0.0;
      if (tri_ok(ii, jj)) {
        v = diff_tbar_gathered(kh, y, ii, jj, k, l, d, t);
        if (t == 0 && ii == 0 && jj == 0) v = v * (double)cG.pntmask[l * 2 + 0];
        if (t == 1 && ii == 1 && jj == 0)
          v = v + diff_tbar_gathered(kh, y, 0, 0, k, l, d, 0) * (double)cG.pntmask[l * 2 + 1];
      }
      tb[(t * 3 + d) * n + p] = v;
    }
}

// per point: the cotangent of s from the triangles that hold it
__global__ void k_diff_adj_pt(const double* tb, double* g) {
  const int p = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (p >= cD.npti) return;
  const int G = cD.G, KA = cD.KA, n = cD.npti;
  const int i = p % G, j = (p / G) % G, k = (p / (G * G)) % KA, l = p / (G * G * KA);
  // (triangle offset, kind t, vertex m): s(i,j) is vertex 1 of TI / TJ (i,j), vertex 2 of TI (i-1,j),
  // vertex 3 of TI (i-1,j-1), vertex 2 of TJ (i-1,j-1), vertex 3 of TJ (i,j-1)
  const int oi[6] = {0, 0, -1, -1, -1, 0}, oj[6] = {0, 0, 0, -1, -1, -1};
  const int tt[6] = {0, 1, 0, 0, 1, 1}, mm[6] = {0, 0, 1, 2, 1, 2};
  double acc = 0.0;
  for (int c = 0; c < 6; ++c) {
    const int ii = i + oi[c], jj = j + oj[c];
    if (!tri_ok(ii, jj)) continue;
    const int q = ix(ii, jj, k, l);
    for (int d = 0; d < 3; ++d)
      acc += P2(cG.intp_w, (d * 3 + mm[c]) * 2 + tt[c], ii, jj, l) * div3(tb[(tt[c] * 3 + d) * n + q]);
  }
  g[p] = acc;
}

// the pole row's adjoint: the pole point and its five ring points
__global__ void k_diff_adj_pl(const double* kh, const double* y, double* g) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP;
  const double y0 = y[ipl(0, k, lp)];
  const double khn = kh[ipl(0, k, lp)];
  double vtb[5][3] = {};
  for (int v = 1; v <= 5; ++v) {
    const int vm1 = (v == 1) ? 5 : v - 1;
    const double kavg = 0.5 * (khn + kh[ipl(v, k, lp)]);
    for (int d = 0; d < 3; ++d) {
      const double w = y0 * kavg * cG.coef_diff_pl[(v * cD.LP + lp) * 3 + d];
      vtb[vm1 - 1][d] += w;
      vtb[v - 1][d] += w;
    }
  }
  double gs[6] = {};
  for (int v = 1; v <= 5; ++v) {
    const int vp1 = (v == 5) ? 1 : v + 1;
    for (int d = 0; d < 3; ++d) {
      const double* cI = cG.coef_intp_pl + ((v * cD.LP + lp) * 3 + d) * 3;
      const double c0 = cI[0], c1 = cI[1], c2 = cI[2];
      const double b = div3(vtb[v - 1][d]);
      gs[0] += (2.0 * c0 - c1 - c2) * b;
      gs[v] += (-c0 + 2.0 * c1 - c2) * b;
      gs[vp1] += (-c0 - c1 + 2.0 * c2) * b;
    }
  }
  for (int g_ = 0; g_ < 6; ++g_) g[ipl(g_, k, lp)] = gs[g_];
}

// ---------------------------------------------------------------------------
// Divergence damping (mod_numfilter.py:2032-2268): the 3-D operator
// OPRT3D_divdamp (kernels/oprt3ddivdamp.py:50-237) of the four momenta
// (rhogvx, rhogvy, rhogvz, rhogw) and the 2-D OPRT_divdamp
// (kernels/oprtdivdamp.py:54-173) of three components, each after the halo
// exchange of its inputs, and their adjoints.  Per triangle the scalar
//   T = sum over directions and vertices of coef_intp x v  (+ the vertical
//       flux difference ((rwv(k+1) at the vertices) - (rwv(k))) / 3 rdgz(k)
//       in 3-D, rwv the half-level mass flux of fluxconv's rhogw_vmh),
// the 3-D operator with the singular-point fix at (0,0); each cell sums
// coef_diff x (T + T') over its six edges per direction.  The 3-D outputs
// live on kmin..kmax, the 2-D on every level.  The adjoint gathers for every
// triangle the edge weights of the cells that use it, then for every point
// the weights of the triangles that hold it (and, in 3-D, the vertical flux's
// weights at levels k and k + 1).
// ---------------------------------------------------------------------------
// the half-level vertical mass flux at point q, level k (zero outside kmin+1..kmax)
__device__ __forceinline__ double dd_rwv(const double* v, int q, int k) {
  if (k < cD.kmin + 1 || k > cD.kmax) return 0.0;
  const int n = cD.npti, qm = q - cD.planei;
  const double* cz = cG.C2WGz;
  const double h = cz[q] * v[q] + cz[n + q] * v[qm] + cz[2 * n + q] * v[n + q] + cz[3 * n + q] * v[n + qm] +
                   cz[4 * n + q] * v[2 * n + q] + cz[5 * n + q] * v[2 * n + qm];
  return h * gam_at(cG.RGAMH, q) + v[3 * n + q] * cG.RGSQRTH[q];
}
// raw triangle value (kind t: 0 TI, 1 TJ) at level k; 3-D with the vertical term and RGAM
__device__ double dd_tri(const double* v, int ii, int jj, int k, int l, int t, bool three) {
  if (!tri_ok(ii, jj)) return 0.0;
  const int n = cD.npti;
  const int qa = ix(ii, jj, k, l), qc = ix(ii + 1, jj + 1, k, l);
  const int qb = (t == 0) ? ix(ii + 1, jj, k, l) : qc;
  const int q3 = (t == 0) ? qc : ix(ii, jj + 1, k, l);
  double sum = 0.0;
  for (int dir = 0; dir < 3; ++dir) {
    const double* f = v + dir * n;
    const double va = three ? f[qa] * gam_at(cG.RGAM, qa) : f[qa];
    const double vb = three ? f[qb] * gam_at(cG.RGAM, qb) : f[qb];
    const double v3 = three ? f[q3] * gam_at(cG.RGAM, q3) : f[q3];
    const double a = P2(cG.coef_intp, (dir * 3 + 0) * 2 + t, ii, jj, l) * va;
    const double b = P2(cG.coef_intp, (dir * 3 + 1) * 2 + t, ii, jj, l) * vb;
    const double c = P2(cG.coef_intp, (dir * 3 + 2) * 2 + t, ii, jj, l) * v3;
    sum = (dir == 0) ? (a + b) + c : ((sum + a) + b) + c;
  }
  if (three) {
    const double up = (dd_rwv(v, qa + cD.planei, k + 1) + dd_rwv(v, qb + cD.planei, k + 1)) +
                      dd_rwv(v, q3 + cD.planei, k + 1);
    const double dn = (dd_rwv(v, qa, k) + dd_rwv(v, qb, k)) + dd_rwv(v, q3, k);
    sum = sum + div3(up - dn) * cC.rdgz[k];
  }
  return sum;
}
__device__ __forceinline__ double dd_tri_fixed(const double* v, int ii, int jj, int k, int l, int t, bool three) {
  double x = dd_tri(v, ii, jj, k, l, t, three);
  if (three && t == 0 && ii == 0 && jj == 0)
    x = x * (double)cG.pntmask[l * 2 + 0] + dd_tri(v, 1, 0, k, l, 1, three) * (double)cG.pntmask[l * 2 + 1];
  return x;
}
// three: v holds four components (rhogvx, rhogvy, rhogvz, rhogw), else three
__global__ void k_ddamp_fwd(const double* v, double* y, int three) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.npti) return;
  const int G = cD.G, KA = cD.KA, n = cD.npti;
  const int i = t % G, j = (t / G) % G, k = (t / (G * G)) % KA, l = t / (G * G * KA);
  const bool on = interior(i, j) && (!three || (k >= cD.kmin && k <= cD.kmax));
  double aTI = 0.0, aTJ = 0.0, bTI = 0.0, cTI = 0.0, cTJ = 0.0, dTJ = 0.0;
  if (on) {
    aTI = dd_tri_fixed(v, i, j, k, l, 0, three);
    aTJ = dd_tri_fixed(v, i, j, k, l, 1, three);
    bTI = dd_tri_fixed(v, i - 1, j, k, l, 0, three);
    cTI = dd_tri_fixed(v, i - 1, j - 1, k, l, 0, three);
    cTJ = dd_tri_fixed(v, i - 1, j - 1, k, l, 1, three);
    dTJ = dd_tri_fixed(v, i, j - 1, k, l, 1, three);
  }
  for (int d = 0; d < 3; ++d) {
    double o = 0.0;
    if (on) {
      auto cd = [&](int e) { return P2(cG.coef_diff, d * 6 + e, i, j, l); };
      o = cd(0) * (aTI + aTJ) + cd(1) * (aTJ + bTI) + cd(2) * (bTI + cTJ) + cd(3) * (cTJ + cTI) +
          cd(4) * (cTI + dTJ) + cd(5) * (dTJ + aTI);
    }
    y[d * n + t] = o;
  }
}

// pole rows: the pole point from its five triangles; ring rows zero
__device__ __forceinline__ double dd_rwv_pl(const double* v, int g, int k, int lp) {
  if (k < cD.kmin + 1 || k > cD.kmax) return 0.0;
  const int np = cD.npl, q = ipl(g, k, lp), qm = ipl(g, k - 1, lp);
  const double* cz = cG.C2WGz_pl + q * 6;
  const double h = cz[0] * v[q] + cz[1] * v[qm] + cz[2] * v[np + q] + cz[3] * v[np + qm] + cz[4] * v[2 * np + q] +
                   cz[5] * v[2 * np + qm];
  return h * gam_at(cG.RGAMH_pl, q) + v[3 * np + q] * cG.RGSQRTH_pl[q];
}
__global__ void k_ddamp_fwd_pl(const double* v, double* y, int three) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP, np = cD.npl;
  for (int g = 0; g < 6; ++g)
    for (int d = 0; d < 3; ++d) y[d * np + ipl(g, k, lp)] = 0.0;
  if (three && (k < cD.kmin || k > cD.kmax)) return;
  double vm[6][3];
  for (int g = 0; g < 6; ++g) {
    const int q = ipl(g, k, lp);
    for (int d = 0; d < 3; ++d) vm[g][d] = three ? v[d * np + q] * gam_at(cG.RGAM_pl, q) : v[d * np + q];
  }
  double sclt[5];
  for (int vv = 1; vv <= 5; ++vv) {
    const int vp1 = (vv == 5) ? 1 : vv + 1;
    const double* cI = cG.coef_intp_pl + (vv * cD.LP + lp) * 9;
    double x = cI[0] * vm[0][0] + cI[1] * vm[vv][0] + cI[2] * vm[vp1][0] + cI[3] * vm[0][1] + cI[4] * vm[vv][1] +
               cI[5] * vm[vp1][1] + cI[6] * vm[0][2] + cI[7] * vm[vv][2] + cI[8] * vm[vp1][2];
    if (three) {
      const double up = (dd_rwv_pl(v, 0, k + 1, lp) + dd_rwv_pl(v, vv, k + 1, lp)) + dd_rwv_pl(v, vp1, k + 1, lp);
      const double dn = (dd_rwv_pl(v, 0, k, lp) + dd_rwv_pl(v, vv, k, lp)) + dd_rwv_pl(v, vp1, k, lp);
      x = x + div3(up - dn) * cC.rdgz[k];
    }
    sclt[vv - 1] = x;
  }
  for (int d = 0; d < 3; ++d) {
    double row = 0.0;
    for (int vv = 1; vv <= 5; ++vv) {
      const int vm1 = (vv == 1) ? 5 : vv - 1;
      const double tv = cG.coef_diff_pl[(vv * cD.LP + lp) * 3 + d] * (sclt[vm1 - 1] + sclt[vv - 1]);
      row = (vv == 1) ? tv : row + tv;
    }
    y[d * np + ipl(0, k, lp)] = row;
  }
}

// cotangent of a raw triangle value from the cells that use it (three directions)
__device__ double dd_tbar_gathered(const double* y, int ii, int jj, int k, int l, int t) {
  const int n = cD.npti;
  const int ci[3] = {ii, ii + 1, t == 0 ? ii + 1 : ii};
  const int cj[3] = {jj, t == 0 ? jj : jj + 1, jj + 1};
  const int e0[3] = {0, t == 0 ? 1 : 2, t == 0 ? 3 : 4};
  const int e1[3] = {t == 0 ? 5 : 1, t == 0 ? 2 : 3, t == 0 ? 4 : 5};
  double acc = 0.0;
  for (int c = 0; c < 3; ++c) {
    const int i = ci[c], j = cj[c];
    if (i < 1 || j < 1 || i > cD.G - 2 || j > cD.G - 2) continue;
    const int q = ix(i, j, k, l);
    for (int d = 0; d < 3; ++d)
      acc += y[d * n + q] * (P2(cG.coef_diff, d * 6 + e0[c], i, j, l) + P2(cG.coef_diff, d * 6 + e1[c], i, j, l));
  }
  return acc;
}
// per triangle point and level: the cotangents of its two raw triangle values
// (tb[t * npt + point]); zero outside the levels the operator writes
__global__ void k_ddamp_adj_tri(const double* y, double* tb, int three) {
  const int p = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (p >= cD.npti) return;
  const int G = cD.G, KA = cD.KA, n = cD.npti;
  const int ii = p % G, jj = (p / G) % G, k = (p / (G * G)) % KA, l = p / (G * G * KA);
  const bool lev = !three || (k >= cD.kmin && k <= cD.kmax);
  for (int t = 0; t < 2; ++t) {
    double v = 0.0;
    if (lev && tri_ok(ii, jj)) {
      v = dd_tbar_gathered(y, ii, jj, k, l, t);
      if (three && t == 0 && ii == 0 && jj == 0) v = v * (double)cG.pntmask[l * 2 + 0];
      if (three && t == 1 && ii == 1 && jj == 0)
        v = v + dd_tbar_gathered(y, 0, 0, k, l, 0) * (double)cG.pntmask[l * 2 + 1];
    }
    tb[t * n + p] = v;
  }
}
// sum over the triangles holding point (i, j) at level k of weight(t, vertex, ii, jj) x tb
template <class W>
__device__ __forceinline__ double dd_gather_pt(const double* tb, int i, int j, int k, int l, W w) {
  const int oi[6] = {0, 0, -1, -1, -1, 0}, oj[6] = {0, 0, 0, -1, -1, -1};
  const int tt[6] = {0, 1, 0, 0, 1, 1}, mm[6] = {0, 0, 1, 2, 1, 2};
  double acc = 0.0;
  for (int c = 0; c < 6; ++c) {
    const int ii = i + oi[c], jj = j + oj[c];
    if (!tri_ok(ii, jj)) continue;
    acc += w(tt[c], mm[c], ii, jj) * tb[tt[c] * cD.npti + ix(ii, jj, k, l)];
  }
  return acc;
}
// the 3-D vertical flux's cotangent at point (i, j), half level kp
__device__ double dd_rwvbar(const double* tb, int i, int j, int kp, int l) {
  if (kp < cD.kmin + 1 || kp > cD.kmax) return 0.0;
  auto one = [](int, int, int, int) { return 1.0; };
  const double up = dd_gather_pt(tb, i, j, kp - 1, l, one) * cC.rdgz[kp - 1] / 3.0;
  const double dn = dd_gather_pt(tb, i, j, kp, l, one) * cC.rdgz[kp] / 3.0;
  return up - dn;
}
// per point: the inputs' cotangents (three components, and rhogw in 3-D)
__global__ void k_ddamp_adj_pt(const double* tb, double* g, int three) {
  const int p = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (p >= cD.npti) return;
  const int G = cD.G, KA = cD.KA, n = cD.npti;
  const int i = p % G, j = (p / G) % G, k = (p / (G * G)) % KA, l = p / (G * G * KA);
  const bool lev = !three || (k >= cD.kmin && k <= cD.kmax);
  double r0 = 0.0, r1 = 0.0;
  if (three) {
    r0 = dd_rwvbar(tb, i, j, k, l);
    r1 = (k + 1 < KA) ? dd_rwvbar(tb, i, j, k + 1, l) : 0.0;
  }
  for (int dir = 0; dir < 3; ++dir) {
    double acc = 0.0;
    if (lev) {
      acc = dd_gather_pt(tb, i, j, k, l, [&](int t, int m, int ii, int jj) {
        return P2(cG.coef_intp, (dir * 3 + m) * 2 + t, ii, jj, l);
      });
      if (three) acc = acc * gam_at(cG.RGAM, p);
    }
    if (three) {
      const int n6 = cD.npti;
      if (r0 != 0.0) acc += r0 * gam_at(cG.RGAMH, p) * cG.C2WGz[(2 * dir) * n6 + p];
      if (r1 != 0.0) {
        const int pu = p + cD.planei;
        acc += r1 * gam_at(cG.RGAMH, pu) * cG.C2WGz[(2 * dir + 1) * n6 + pu];
      }
    }
    g[dir * n + p] = acc;
  }
  if (three) g[3 * n + p] = r0 * cG.RGSQRTH[p];
}
// the pole rows' adjoint (one thread per level and pole)
__global__ void k_ddamp_adj_pl(const double* y, double* g, int three) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP, np = cD.npl, KA = cD.KA;
  const int nc = three ? 4 : 3;
  // the triangles' cotangents at level kk (zero where the operator writes nothing)
  auto sbar = [&](int kk, double out[5]) {
    for (int vv = 0; vv < 5; ++vv) out[vv] = 0.0;
    if (kk < 0 || kk >= KA || (three && (kk < cD.kmin || kk > cD.kmax))) return;
    for (int vv = 1; vv <= 5; ++vv) {
      const int vp1 = (vv == 5) ? 1 : vv + 1;
      double acc = 0.0;
      for (int d = 0; d < 3; ++d)
        acc += y[d * np + ipl(0, kk, lp)] *
               (cG.coef_diff_pl[(vv * cD.LP + lp) * 3 + d] + cG.coef_diff_pl[(vp1 * cD.LP + lp) * 3 + d]);
      out[vv - 1] = acc;
    }
  };
  double sb[5];
  sbar(k, sb);
  double gv[6][4] = {};
  for (int vv = 1; vv <= 5; ++vv) {
    const int vp1 = (vv == 5) ? 1 : vv + 1;
    const double* cI = cG.coef_intp_pl + (vv * cD.LP + lp) * 9;
    for (int d = 0; d < 3; ++d) {
      gv[0][d] += cI[d * 3 + 0] * sb[vv - 1];
      gv[vv][d] += cI[d * 3 + 1] * sb[vv - 1];
      gv[vp1][d] += cI[d * 3 + 2] * sb[vv - 1];
    }
  }
  if (three) {
    for (int g_ = 0; g_ < 6; ++g_)
      for (int d = 0; d < 3; ++d) gv[g_][d] = gv[g_][d] * gam_at(cG.RGAM_pl, ipl(g_, k, lp));
    // the vertical flux's cotangent at pole point g_, half level kp: the triangles holding g_
    auto rbar = [&](int g_, int kp) {
      if (kp < cD.kmin + 1 || kp > cD.kmax) return 0.0;
      double su[5], sd[5];
      sbar(kp - 1, su);
      sbar(kp, sd);
      double up = 0.0, dn = 0.0;
      for (int vv = 1; vv <= 5; ++vv) {
        const int vp1 = (vv == 5) ? 1 : vv + 1;
        if (g_ == 0 || g_ == vv || g_ == vp1) {
          up += su[vv - 1];
          dn += sd[vv - 1];
        }
      }
      return up * cC.rdgz[kp - 1] / 3.0 - dn * cC.rdgz[kp] / 3.0;
    };
    for (int g_ = 0; g_ < 6; ++g_) {
      const double r0 = rbar(g_, k), r1 = (k + 1 < KA) ? rbar(g_, k + 1) : 0.0;
      const int q = ipl(g_, k, lp);
      for (int d = 0; d < 3; ++d) {
        if (r0 != 0.0) gv[g_][d] += r0 * gam_at(cG.RGAMH_pl, q) * cG.C2WGz_pl[q * 6 + 2 * d];
        if (r1 != 0.0) {
          const int qu = ipl(g_, k + 1, lp);
          gv[g_][d] += r1 * gam_at(cG.RGAMH_pl, qu) * cG.C2WGz_pl[qu * 6 + 2 * d + 1];
        }
      }
      gv[g_][3] = r0 * cG.RGSQRTH_pl[q];
    }
  }
  for (int g_ = 0; g_ < 6; ++g_)
    for (int c = 0; c < nc; ++c) g[c * np + ipl(g_, k, lp)] = gv[g_][c];
}

// ---------------------------------------------------------------------------
// The Kh-weighted diffusion's dependence on its coefficient field: y is
// bilinear in (s, kh) through the edge weights kf_e = (kh(cell) + kh(edge
// neighbour e)) / 2, so d<ybar, y>/d kh gathers, for every point, half of
// ybar x E_e at the cells whose weight kf_e it enters (as the cell itself, or
// as the neighbour across edge e), E_e = sum over directions of coef_diff x
// the edge's pair of (fixed) triangle values of the exchanged s.
// ---------------------------------------------------------------------------
__device__ void diff_edge_sums(const double* s, int i, int j, int k, int l, double E[6]) {
  for (int e = 0; e < 6; ++e) E[e] = 0.0;
  for (int d = 0; d < 3; ++d) {
    const double aTI = diff_tri_fixed(s, i, j, k, l, d, 0), aTJ = diff_tri_fixed(s, i, j, k, l, d, 1);
    const double bTI = diff_tri_fixed(s, i - 1, j, k, l, d, 0);
    const double cTI = diff_tri_fixed(s, i - 1, j - 1, k, l, d, 0), cTJ = diff_tri_fixed(s, i - 1, j - 1, k, l, d, 1);
    const double dTJ = diff_tri_fixed(s, i, j - 1, k, l, d, 1);
    const double pr[6] = {aTI + aTJ, aTJ + bTI, bTI + cTJ, cTJ + cTI, cTI + dTJ, dTJ + aTI};
    for (int e = 0; e < 6; ++e) E[e] += P2(cG.coef_diff, d * 6 + e, i, j, l) * pr[e];
  }
}
__global__ void k_diff_khbar(const double* s, const double* y, double* gkh) {
  const int p = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (p >= cD.npti) return;
  const int G = cD.G, KA = cD.KA;
  const int i = p % G, j = (p / G) % G, k = (p / (G * G)) % KA, l = p / (G * G * KA);
  // the edge-e neighbour of cell (i, j) is (i + oi[e], j + oj[e]) (the order of diff_kf)
  const int oi[6] = {1, 0, -1, -1, 0, 1}, oj[6] = {1, 1, 0, -1, -1, 0};
  double E[6], acc = 0.0;
  if (interior(i, j)) {
    diff_edge_sums(s, i, j, k, l, E);
    const double yp = y[ix(i, j, k, l)];
    for (int e = 0; e < 6; ++e) acc += 0.5 * yp * E[e];
  }
  for (int e = 0; e < 6; ++e) {
    const int ci = i - oi[e], cj = j - oj[e];
    if (ci < 1 || cj < 1 || ci > G - 2 || cj > G - 2) continue;
    diff_edge_sums(s, ci, cj, k, l, E);
    acc += 0.5 * y[ix(ci, cj, k, l)] * E[e];
  }
  gkh[p] = acc;
}
__global__ void k_diff_khbar_pl(const double* s, const double* y, double* gkh) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  const int k = t / cD.LP, lp = t % cD.LP;
  const double sn = s[ipl(0, k, lp)], y0 = y[ipl(0, k, lp)];
  double vt[5][3];
  for (int v = 1; v <= 5; ++v) {
    const int vp1 = (v == 5) ? 1 : v + 1;
    const double sij = s[ipl(v, k, lp)], sp1 = s[ipl(vp1, k, lp)];
    for (int d = 0; d < 3; ++d) {
      const double* cI = cG.coef_intp_pl + ((v * cD.LP + lp) * 3 + d) * 3;
      const double c0 = cI[0], c1 = cI[1], c2 = cI[2];
      vt[v - 1][d] = div3((2.0 * c0 - c1 - c2) * sn + (-c0 + 2.0 * c1 - c2) * sij + (-c0 - c1 + 2.0 * c2) * sp1);
    }
  }
  double g0 = 0.0;
  gkh[ipl(0, k, lp)] = 0.0;
  for (int v = 1; v <= 5; ++v) {
    const int vm1 = (v == 1) ? 5 : v - 1;
    double sd = 0.0;
    for (int d = 0; d < 3; ++d) sd += cG.coef_diff_pl[(v * cD.LP + lp) * 3 + d] * (vt[vm1 - 1][d] + vt[v - 1][d]);
    g0 += 0.5 * y0 * sd;
    gkh[ipl(v, k, lp)] = 0.5 * y0 * sd;
  }
  gkh[ipl(0, k, lp)] = g0;
}

}  // namespace nc
