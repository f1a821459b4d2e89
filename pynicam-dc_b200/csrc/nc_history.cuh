// Derived history diagnostics on the device: Hvar.history_vars
// (pynicamdc/nhm/driver/mod_history_vars.py:30-186) as Dyn.history_vars_step
// (pynicamdc/nhm/dynamics/mod_dynamics.py:737-772) calls it, on the state the
// handle holds.  The diagnostic state is re-derived from the prognostic with
// the step's own expressions (kernels/diag.py:53-143); the half-level w outside
// kmin+1..kmax comes from the diagnostic w the last step left (the reference
// reads those rows from its persistent DIAG buffer) through the reference's
// filter.  Every output is written for all (i, j), halo included, like the
// reference's full arrays.  log, pow, exp and cos are CUDA's, so the
// thermodynamic ratios, saturation ratios and pressure-level slices can differ
// from numpy in the last bit; the rest uses the reference's association order.
#pragma once
#include "nc_ops.cuh"

namespace nc {

// item ids: the reference's model-level names in its I/O order
// (share/mod_io.py:251-257), then the 2-D ones (:258-260)
enum HistItem {
  H_U, H_V, H_W, H_TH, H_THV, H_OMG, H_PRES, H_TEM, H_RHO, H_HGT, H_MSE, H_RH, H_RHA, H_RHI,
  H_DU, H_DV, H_DW, H_DTEM, H_DQ, H_UCOS, H_VCOS, H_TH_PRIME,
  H_PS, H_PW, H_LWP, H_IWP,
  H_SL0,                 // then for 850, 500, 250, 100 hPa: u, v, w, t
  H_CL = H_SL0 + 16,     // the terminator chemistry's column means (AF_TYPE 'DCMIP' only): Cl, Cl2, Cly
  H_CL2, H_CLY,
  H_N
};
constexpr int H_N3 = H_PS;   // ids below are (i, j, k, l) fields, the rest (i, j, l)

struct HistArgs {
  const double* P[6];       // RHOG, RHOGVX, RHOGVY, RHOGVZ, RHOGW, RHOGE
  const double* Pq[NC_MAXNQ];
  int iqv;                  // water-vapour tracer (-1: none)
  int iql[2], iqs[3];       // liquid (QC, QR) and solid (QI, QS, QG) tracers (-1: absent)
  int icl, icl2;            // the chemistry's Cl and Cl2 tracers (-1: none)
  const double* wdiag;      // diagnostic w of the last step [l][k][j][i]
  const double *hgt, *coslat, *zsfc, *IJ;   // GRD_Z [l][k][j][i]; planes [l][j][i]; IJ [6][l][j][i]
  const double* dgz;        // GRD_dgz (kall)
  const double* thmean;     // per-level area-weighted mean of th (kall)
  double* out[H_N];         // device outputs, null where not requested
  double* old[5];           // previous u, v, wc, tem, qv of the tendency fields
  int tform[5];             // per tendency: 0 zero (no earlier output of it), 1 (old - cur) * fac / dn
  double fac, fac_q, dn;    // 86400/dt, 86400/dt*1e3, steps since the last output
  double LHV, UNDEF, PSAT0, RTEM00, CPovR_liq, CPovR_ice, LovR_liq, LovR_ice, SAT_LL, SAT_UL;
};

// the diagnostic state at one level of a regional column (kernels/diag.py:88-115)
struct DiagPt {
  double rho, vx, vy, vz, tem, pre, qv;
};
__device__ __forceinline__ DiagPt hist_diag(const HistArgs& a, int p) {
  DiagPt d;
  const double RHOG = a.P[0][p];
  d.rho = RHOG / cG.GSGAM2[p];
  const Recip rr = recip_of(RHOG);
  d.vx = div_by(a.P[1][p], rr);
  d.vy = div_by(a.P[2][p], rr);
  d.vz = div_by(a.P[3][p], rr);
  const double ein = div_by(a.P[5][p], rr);
  const double q0 = div_by(a.Pq[0][p], rr);
  double qd, cv;
  moist_qd_cv([&](int n) { return div_by(a.Pq[n][p], rr); }, q0, qd, cv);
  d.tem = ein / cv;
  d.pre = d.rho * d.tem * (qd * cC.Rdry + q0 * cC.Rvap);
  d.qv = (a.iqv >= 0) ? div_by(a.Pq[a.iqv][p], rr) : 0.0;
  return d;
}

// half-level w at level k of the column (base q0): the interior levels from the
// prognostic, the others from the last step's diagnostic buffer, filtered
// (mod_history_vars.py:74-75)
__device__ __forceinline__ double hist_w(const HistArgs& a, int q0, int k) {
  const int kmin = cD.kmin, kmax = cD.kmax, ks = cD.planei;
  const int p = q0 + k * ks;
  double w;
  if (k >= kmin + 1 && k <= kmax) {
    const int pm = p - ks;
    w = a.P[4][p] / (cG.C2W[p] * a.P[0][p] + cG.C2W[cD.npti + p] * a.P[0][pm]);
  } else {
    w = a.wdiag[p];
  }
  const bool keep = isfinite(w) && (fabs(w) < fabs(a.UNDEF) * 0.1);
  return keep ? w : 0.0;
}

// cell-centre w (mod_history_vars.py:76-80): zero outside kmin..kmax
__device__ __forceinline__ double hist_wc(const HistArgs& a, int q0, int k) {
  if (k < cD.kmin || k > cD.kmax) return 0.0;
  const int p = q0 + k * cD.planei;
  return cG.W2C[p] * hist_w(a, q0, k + 1) + cG.W2C[cD.npti + p] * hist_w(a, q0, k);
}

// saturation vapour pressures (nhm/share/mod_saturation.py:83-98)
__device__ __forceinline__ double psat_liq(const HistArgs& a, double t) {
  return a.PSAT0 * pow(t * a.RTEM00, a.CPovR_liq) * exp(a.LovR_liq * (a.RTEM00 - 1.0 / t));
}
__device__ __forceinline__ double psat_ice(const HistArgs& a, double t) {
  return a.PSAT0 * pow(t * a.RTEM00, a.CPovR_ice) * exp(a.LovR_ice * (a.RTEM00 - 1.0 / t));
}

__device__ __forceinline__ double hist_th(const DiagPt& d) {
  return d.tem * pow(cC.PRE00 / d.pre, cC.Rdry / cC.CPdry);   // THRMDYN_th (share/mod_thrmdyn.py:247-262)
}

// One thread per regional column (i, j, l), halo included.
__global__ void __launch_bounds__(128) k_history(HistArgs a) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.npt2i) return;
  const int G = cD.G, KA = cD.KA, kmin = cD.kmin, kmax = cD.kmax, ks = cD.planei;
  const int i = t % G, j = (t / G) % G, l = t / (G * G);
  const int q0 = ix(i, j, 0, l);
  const int c2 = (l * G + j) * G + i;   // plane index [l][j][i]
  const int np2 = cD.npt2i;
  const double GRAV = cC.GRAV;
  const double IX = a.IJ[c2], IY = a.IJ[np2 + c2], IZ = a.IJ[2 * np2 + c2];
  const double JX = a.IJ[3 * np2 + c2], JY = a.IJ[4 * np2 + c2], JZ = a.IJ[5 * np2 + c2];
  const double cosl = a.coslat ? a.coslat[c2] : 1.0;
  double pw = 0.0, lwp = 0.0, iwp = 0.0, rdz = 0.0, ccl = 0.0, ccl2 = 0.0, ccly = 0.0;
  double pre_col[NC_MAXK];
  for (int k = 0; k < KA; ++k) {
    const int p = q0 + k * ks;
    const DiagPt d = hist_diag(a, p);
    pre_col[k] = d.pre;
    const double hu = d.vx * IX + d.vy * IY + d.vz * IZ;
    const double hv = d.vx * JX + d.vy * JY + d.vz * JZ;
    const double wc = hist_wc(a, q0, k);
    const double hgt = a.hgt[p];
    if (a.out[H_RHO]) a.out[H_RHO][p] = d.rho;
    if (a.out[H_TEM]) a.out[H_TEM][p] = d.tem;
    if (a.out[H_PRES]) a.out[H_PRES][p] = d.pre;
    if (a.out[H_HGT]) a.out[H_HGT][p] = hgt;
    if (a.out[H_U]) a.out[H_U][p] = hu;
    if (a.out[H_V]) a.out[H_V][p] = hv;
    if (a.out[H_W]) a.out[H_W][p] = wc;
    if (a.out[H_OMG]) a.out[H_OMG][p] = -GRAV * d.rho * wc;
    if (a.out[H_TH] || a.out[H_THV] || a.out[H_TH_PRIME]) {
      const double th = hist_th(d);
      if (a.out[H_TH]) a.out[H_TH][p] = th;
      if (a.out[H_THV]) a.out[H_THV][p] = (a.iqv >= 0) ? th * (1.0 + 0.61 * d.qv) : th;
      if (a.out[H_TH_PRIME]) a.out[H_TH_PRIME][p] = th - a.thmean[k];
    }
    if (a.out[H_UCOS]) a.out[H_UCOS][p] = hu * cosl;
    if (a.out[H_VCOS]) a.out[H_VCOS][p] = hv * cosl;
    if (a.out[H_MSE]) a.out[H_MSE][p] = d.tem * cC.CPdry + hgt * GRAV + d.qv * a.LHV;
    if (a.out[H_RH] || a.out[H_RHA] || a.out[H_RHI]) {
      const double num = d.qv * d.rho * cC.Rvap * d.tem * 100.0;
      const double pl = psat_liq(a, d.tem), pi = psat_ice(a, d.tem);
      if (a.out[H_RH]) a.out[H_RH][p] = num / pl;
      if (a.out[H_RHI]) a.out[H_RHI][p] = num / pi;
      if (a.out[H_RHA]) {
        const double al = fmin(fmax((d.tem - a.SAT_LL) / (a.SAT_UL - a.SAT_LL), 0.0), 1.0);
        a.out[H_RHA][p] = num / (pl * al + pi * (1.0 - al));
      }
    }
    // interval tendencies (mod_history_vars.py:166-180)
    const double cur[5] = {hu, hv, wc, d.tem, d.qv};
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      double* o = a.out[H_DU + n];
      if (!o) continue;
      const double fac = (n == 4) ? a.fac_q : a.fac;
      o[p] = a.tform[n] ? (a.old[n][p] - cur[n]) * fac / a.dn : 0.0;
      a.old[n][p] = cur[n];
    }
    // column integrals over kmin..kmax (mod_history_vars.py:138-157)
    if (k >= kmin && k <= kmax) {
      const double wcol = cG.GSGAM2[p] * a.dgz[k];
      const double RHOG = a.P[0][p];
      double ql = 0.0, qs = 0.0;
      for (int m = 0; m < 2; ++m)
        if (a.iql[m] >= 0) ql = ql + a.Pq[a.iql[m]][p] / RHOG;
      for (int m = 0; m < 3; ++m)
        if (a.iqs[m] >= 0) qs = qs + a.Pq[a.iqs[m]][p] / RHOG;
      const double xv = d.rho * d.qv * wcol, xl = d.rho * ql * wcol, xs = d.rho * qs * wcol;
      pw = (k == kmin) ? xv : pw + xv;
      lwp = (k == kmin) ? xl : lwp + xl;
      iwp = (k == kmin) ? xs : iwp + xs;
      if (a.icl >= 0) {   // mod_history_vars.py:149-156
        const double q1 = a.Pq[a.icl][p] / RHOG, q2 = a.Pq[a.icl2][p] / RHOG;
        const double xo = d.rho * 1.0 * wcol, x1 = d.rho * q1 * wcol, x2 = d.rho * q2 * wcol;
        const double x3 = d.rho * (q1 + 2.0 * q2) * wcol;
        rdz = (k == kmin) ? xo : rdz + xo;
        ccl = (k == kmin) ? x1 : ccl + x1;
        ccl2 = (k == kmin) ? x2 : ccl2 + x2;
        ccly = (k == kmin) ? x3 : ccly + x3;
      }
    }
    if (k == kmin && a.out[H_PS]) a.out[H_PS][c2] = d.pre + d.rho * GRAV * (hgt - a.zsfc[c2]);
  }
  if (a.out[H_PW]) a.out[H_PW][c2] = pw;
  if (a.out[H_LWP]) a.out[H_LWP][c2] = lwp;
  if (a.out[H_IWP]) a.out[H_IWP][c2] = iwp;
  if (a.out[H_CL]) a.out[H_CL][c2] = ccl / rdz;
  if (a.out[H_CL2]) a.out[H_CL2][c2] = ccl2 / rdz;
  if (a.out[H_CLY]) a.out[H_CLY][c2] = ccly / rdz;
  // pressure-level slices, log-p linear between the bracketing levels
  // (mod_history_vars.py:188-209)
  const double plevs[4] = {850.0e2, 500.0e2, 250.0e2, 100.0e2};
  for (int s = 0; s < 4; ++s) {
    if (!(a.out[H_SL0 + 4 * s] || a.out[H_SL0 + 4 * s + 1] || a.out[H_SL0 + 4 * s + 2] || a.out[H_SL0 + 4 * s + 3]))
      continue;
    const double plev = plevs[s];
    int ku = 0;
    for (int k = kmin; k < KA; ++k)
      if (pre_col[k] < plev) {
        ku = k;
        break;
      }
    ku = ku > kmin ? ku : kmin;
    const int kl = ku - 1;
    const DiagPt du = hist_diag(a, q0 + ku * ks), dl = hist_diag(a, q0 + kl * ks);
    const double lpu = log(du.pre), lpl = log(dl.pre), lp = log(plev);
    const double denom = lpl - lpu;
    const double wl = (lp - lpu) / denom, wu = (lpl - lp) / denom;
    const double f_l[4] = {dl.vx * IX + dl.vy * IY + dl.vz * IZ, dl.vx * JX + dl.vy * JY + dl.vz * JZ,
                           hist_wc(a, q0, kl), dl.tem};
    const double f_u[4] = {du.vx * IX + du.vy * IY + du.vz * IZ, du.vx * JX + du.vy * JY + du.vz * JZ,
                           hist_wc(a, q0, ku), du.tem};
#pragma unroll
    for (int f = 0; f < 4; ++f)
      if (a.out[H_SL0 + 4 * s + f]) a.out[H_SL0 + 4 * s + f][c2] = wl * f_l[f] + wu * f_u[f];
  }
}

// Per-level area-weighted mean of th over the interior cells of every region
// (mod_history_vars.py:103-115: sum th * GMTR_area / RGAM^2 over the sum of the
// weights; the pole cells are left out, as there).  One block per level.
__global__ void __launch_bounds__(256) k_history_thmean(HistArgs a, const double* area, double* mean) {
  const int k = (int)blockIdx.x;
  const int G = cD.G, gmin = cD.gmin, n1 = cD.gmax - cD.gmin + 1;
  const int ncell = n1 * n1 * cD.L;
  double sa = 0.0, st = 0.0;
  for (int c = (int)threadIdx.x; c < ncell; c += (int)blockDim.x) {
    const int i = gmin + c % n1, j = gmin + (c / n1) % n1, l = c / (n1 * n1);
    const int p = ix(i, j, k, l);
    const double rg = cG.RGAM[p];
    const double wt = area[(l * G + j) * G + i] / (rg * rg);
    sa += wt;
    st += hist_th(hist_diag(a, p)) * wt;
  }
  __shared__ double ra[256], rt[256];
  ra[threadIdx.x] = sa;
  rt[threadIdx.x] = st;
  __syncthreads();
  for (int s = (int)blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      ra[threadIdx.x] += ra[threadIdx.x + s];
      rt[threadIdx.x] += rt[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) mean[k] = rt[0] / ra[0];
}

// (i, j, l) host layout of a plane [l][j][i]
__global__ void k_pack_plane(double* dst, const double* src) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.npt2i) return;
  const int G = cD.G, L = cD.L;
  const int i = t % G, j = (t / G) % G, l = t / (G * G);
  dst[((long long)i * G + j) * L + l] = src[t];
}

}  // namespace nc
