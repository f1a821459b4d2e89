// Artificial forcing after the dynamics step (Dyn.forcing_step,
// pynicamdc/nhm/dynamics/mod_dynamics.py:597-735): the Held-Suarez case.
#pragma once
#include "nc_small.cuh"

namespace nc {

// Held & Suarez (1994) dry-case parameters (nhm/forcing/mod_af_heldsuarez.py:19-36)
struct HsParams {
  double RdCp;            // Rdry / CPdry
  double sigma_b, Kf, Dth_z, Ka, Ks, T_eq0, DT_y, PRE00;
};
struct HsArgs {
  Prog<double> P;         // PROG, updated in place
  const double* Pqw[NC_MAXQW];   // the water tracers (0: vapour) for the diagnostics
  const double* lat3;     // planes |sin lat|^2, |cos lat|^2, |cos lat|^4 of each column
  double dt;              // large time step
  HsParams hp;
};

// the Held-Suarez tendencies at one level (mod_af_heldsuarez.py:38-88):
// Rayleigh friction below sigma_b and Newtonian relaxation of temperature to
// the radiative-equilibrium profile; psref = (pre(kmin) + pre(kmin-1)) / 2
__device__ __forceinline__ void hs_tendency(const HsParams& a, double sin2, double cos2, double cos4, double psref,
                                            double pre, double tem, double vx, double vy, double vz, double& fvx,
                                            double& fvy, double& fvz, double& fe) {
  const double sigma = pre / psref;
  const double factor = npmax((sigma - a.sigma_b) / (1.0 - a.sigma_b), 0.0);
  fvx = -a.Kf * factor * vx;
  fvy = -a.Kf * factor * vy;
  fvz = -a.Kf * factor * vz;
  const double ap0 = fabs(pre / a.PRE00);
  const double Kt = a.Ka + (a.Ks - a.Ka) * factor * cos4;
  const double T_eq = npmax(200.0, (a.T_eq0 - a.DT_y * sin2 - a.Dth_z * log(npmax(ap0, 1e-30)) * cos2) *
                                       pow(ap0, a.RdCp));
  fe = -Kt * (tem - T_eq) * cC.CVdry;
}

// One thread per interior regional column: the diagnostics of the prognostic
// (kernels/diag.py, no boundary conditions), the Held-Suarez tendencies
// (mod_af_heldsuarez.py:38-88: Rayleigh friction below sigma_b, Newtonian
// relaxation of temperature to the radiative-equilibrium profile; zero
// outside kmin..kmax) and their application PROG + dt * f * rho * GSGAM2 to
// RHOGV{X,Y,Z} and RHOGE, with + 0 on RHOG and RHOGW (mod_forcing.py:14-28).
// Halo columns are left to the exchange that follows; the poles are not
// forced.  Same association order as the reference; log and pow are CUDA's,
// so T_eq can differ from numpy's in the last bits.
__global__ void k_forcing_hs(HsArgs a) {
  const int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l;
  if (!col_of(t, i, j, l) || !interior(i, j)) return;
  const Col c = col_reg(i, j, l);
  const int KA = cD.KA, kmin = cD.kmin, kmax = cD.kmax;
  double* const* P = a.P.v;
  const double sin2 = P2(a.lat3, 0, i, j, l), cos2 = P2(a.lat3, 1, i, j, l), cos4 = P2(a.lat3, 2, i, j, l);
  // diagnostics at level k (kernels/diag.py:53-143)
  auto diag = [&](int k, double& rho, double& pre, double& tem, double& vx, double& vy, double& vz) {
    const int p = c.at(k);
    const double RHOG = P[0][p];
    rho = RHOG / cG.GSGAM2[p];
    vx = P[1][p] / RHOG;
    vy = P[2][p] / RHOG;
    vz = P[3][p] / RHOG;
    const double ein = P[5][p] / RHOG;
    const double q0 = a.Pqw[0][p] / RHOG;
    double qd, cv;
    moist_qd_cv([&](int n) { return a.Pqw[n][p] / RHOG; }, q0, qd, cv);
    tem = ein / cv;
    pre = rho * tem * (qd * cC.Rdry + q0 * cC.Rvap);
  };
  double rho, pre, tem, vx, vy, vz;
  diag(kmin, rho, pre, tem, vx, vy, vz);
  const double pre_kmin = pre;
  diag(kmin - 1, rho, pre, tem, vx, vy, vz);
  const double psref = 0.5 * (pre_kmin + pre);
  for (int k = 0; k < KA; ++k) {
    const int p = c.at(k);
    if (k < kmin || k > kmax) {
#pragma unroll
      for (int v = 0; v < 6; ++v) P[v][p] = P[v][p] + 0.0;
      continue;
    }
    diag(k, rho, pre, tem, vx, vy, vz);
    double fvx, fvy, fvz, fe;
    hs_tendency(a.hp, sin2, cos2, cos4, psref, pre, tem, vx, vy, vz, fvx, fvy, fvz, fe);
    const double gs = cG.GSGAM2[p];
    P[0][p] = P[0][p] + 0.0;
    P[1][p] = P[1][p] + a.dt * fvx * rho * gs;
    P[2][p] = P[2][p] + a.dt * fvy * rho * gs;
    P[3][p] = P[3][p] + a.dt * fvz * rho * gs;
    P[4][p] = P[4][p] + 0.0;
    P[5][p] = P[5][p] + a.dt * fe * rho * gs;
  }
}

// ---------------------------------------------------------------------------
// DCMIP forcing (AF_TYPE 'DCMIP': nhm/forcing/mod_forcing.py:207-321
// forcing_step -> mod_af_dcmip.py:129-317 AF_dcmip): Kessler warm-rain
// microphysics (kessler.py:9-179), the simple physics (simple_physics.py) and
// the terminator toy chemistry, each optional, all from the same state, with
// the Held-Suarez relaxation on top for the moist Held-Suarez case (its
// momentum tendency replaces the others', its energy tendency adds).  One
// thread per regional column (every column of the tile, as the reference
// forces all of them before the exchange): the diagnostics with the water
// tracers vapour, cloud, rain (0, 1, 2), the schemes, the water, momentum and
// energy tendencies (the energy ones from increments), applied as
// PROG + dt * f * rho * GSGAM2 on every level (f zero outside kmin..kmax; the
// water tendencies also added to RHOG), and the column's precipitation rate.
// Same association order as the reference; exp, log, pow, sin, cos are
// CUDA's (sqrt correctly rounded), so results can differ from numpy's in the
// last bits.
// ---------------------------------------------------------------------------
#define NC_KESS_K 64
struct DcmipArgs {
  Prog<double> P;                 // PROG, updated in place
  double* Pq[NC_MAXNQ];           // tracer masses, updated in place
  int nq;
  const double* zf;               // full-level heights [l][k][j][i]
  double* precip;                 // precipitation rate per column [l][j][i]
  double dt, RdCp, PRE00;
  int negative_fixer, update_tot_dens;
  int kessler;                    // Kessler warm-rain microphysics on
  // terminator toy chemistry (optional): the Cl and Cl2 tracer indices, the
  // column latitude and longitude [l][j][i] in radians
  int n_cl, n_cl2;
  const double *lat, *lon;
  // simple physics (optional): large-scale condensation switch, half-level
  // heights [l][k][j][i], surface height, sea-surface temperature [l][j][i],
  // the column unit vectors IX, IY, IZ, JX, JY, JZ [6][l][j][i]
  int sm, sm_lsc, sm_bryan;        // simple physics, its condensation, the Bryan boundary layer
  const double *zh, *zsfc, *tsurf, *ij;
  double sm_C;                    // the heat / moisture exchange coefficient (x4 for moist Held-Suarez)
  // moist Held-Suarez (optional): |sin lat|^2, |cos lat|^2, |cos lat|^4 planes
  int hs;
  const double* hs_lat3;
  HsParams hp;
};

// numpy's sum of a contiguous row (pairwise: eight running partial sums
// combined as ((0+1)+(2+3))+((4+5)+(6+7)), then the remainder in order;
// rows below eight summed in order from 0), for n <= 128
__device__ __forceinline__ double np_rowsum(const double* x, int n) {
  if (n < 8) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s = s + x[i];
    return s;
  }
  double r[8];
  for (int m = 0; m < 8; ++m) r[m] = x[m];
  int i = 8;
  for (; i < n - (n % 8); i += 8)
    for (int m = 0; m < 8; ++m) r[m] = r[m] + x[i + m];
  double s = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
  for (; i < n; ++i) s = s + x[i];
  return s;
}

// DCMIP simple physics (nhm/forcing/simple_physics.py:310-366, the DCMIP2016
// v6 scheme with the RJ2012 boundary layer, or Bryan's with bryan; Cv the exchange coefficient of
// heat and moisture, 0.0011, four times that for moist Held-Suarez) on one column of
// nz levels ordered top to bottom: t, q, u, v updated in place; pm the full-
// level pressure, pint the nz + 1 interface pressures (pint[nz] = ps);
// CE..CFq work arrays of nz.  Returns the large-scale condensation's
// precipitation rate (0 without lsc).  log, exp, pow are CUDA's.
__device__ double simple_physics_col(int nz, double* t, double* q, double* u, double* v, const double* pm,
                                     const double* pint, double ps, double tsurf, double dt, int lsc, double Cv,
                                     int bryan, double* CE, double* CEm, double* CFu, double* CFv, double* CFt,
                                     double* CFq) {
  const double rair = 287.0, rh2o = 461.5, grav = 9.80616, cpair = 1.0045e3, latvap = 2.5e6;
  const double epsilo = rair / rh2o, zvir = (rh2o / rair) - 1.0;
  const double T0 = 273.16, e0 = 610.78, rhow = 1000.0;
  const double Cd0 = 0.0007, Cd1 = 0.000065, Cm = 0.002, v20 = 20.0;
  const double p0 = 100000.0, pbltop = 85000.0, pblconst2 = 10000.0 * 10000.0;
  const int b = nz - 1;
  // height of the lowest full level from the initial state (:73-96)
  const double za = rair / grav * t[b] * (1.0 + zvir * q[b]) * 0.5 * (log(ps) - log(pint[b]));
  double precl = 0.0;
  if (lsc) {   // large-scale condensation (:48-91); the rates into CE for the column sum
    for (int c = 0; c < nz; ++c) {
      const double qsat = epsilo * e0 / pm[c] * exp(-latvap / rh2o * ((1.0 / t[c]) - 1.0 / T0));
      const double denom = 1.0 + (latvap / cpair) * (epsilo * latvap * qsat / (rair * t[c] * t[c]));
      const double cond = (q[c] > qsat) ? (1.0 / dt) * (q[c] - qsat) / denom : 0.0;
      t[c] = t[c] + (latvap / cpair) * cond * dt;
      q[c] = q[c] - cond * dt;
      CE[c] = cond * (pint[c + 1] - pint[c]) / (grav * rhow);
    }
    precl = np_rowsum(CE, nz);
  }
  // drag and diffusivities from the lowest-level wind (:118-149)
  const double wind = sqrt(u[b] * u[b] + v[b] * v[b]);
  const double Cd = (wind < v20) ? Cd0 + Cd1 * wind : Cm;
  const double KmC = Cd * wind * za, KeC = Cv * wind * za;
  auto decay = [&](int c) {
    const double x = pbltop - pint[c];
    return (pint[c] >= pbltop) ? 1.0 : exp(-(x * x) / pblconst2);
  };
  // the Bryan boundary layer (TC_PBL_mod, :128-141): diffusivities from the
  // interface heights below 1 km, integrated upward from the surface
  double kmB[NC_KESS_K], keB[NC_KESS_K];
  if (bryan) {
    double zi = 0.0;
    for (int c = nz - 1; c >= 0; --c) {
      const double dlnpint = log(pint[c + 1]) - log(pint[c]);
      zi = zi + rair / grav * t[c] * (1.0 + zvir * q[c]) * dlnpint;
      const double fac = 1.0 - zi / 1000.0;
      const double base = wind * zi * fac * fac;
      kmB[c] = (zi <= 1000.0) ? 0.4 * sqrt(Cd) * base : 0.0;
      keB[c] = (zi <= 1000.0) ? 0.4 * sqrt(Cv) * base : 0.0;
    }
  }
  // implicit bulk surface fluxes of the lowest level (:200-225)
  const double qsats = epsilo * e0 / ps * exp(-latvap / rh2o * ((1.0 / tsurf) - 1.0 / T0));
  const double dm = 1.0 + Cd * wind * dt / za, dh = 1.0 + Cv * wind * dt / za;
  u[b] = u[b] / dm;
  v[b] = v[b] / dm;
  t[b] = (t[b] + Cv * wind * tsurf * dt / za) / dh;
  q[b] = (q[b] + Cv * wind * qsats * dt / za) / dh;
  // implicit boundary-layer diffusion (:228-307): the interface between c and
  // c + 1 couples them through fm (momentum) and fe (heat, moisture)
  const double kap = rair / cpair, g2dt = dt * grav * grav;
  auto iface = [&](int c, double& fm, double& fe) {
    const double tvp = t[c + 1] * (1.0 + zvir * q[c + 1]), tv = t[c] * (1.0 + zvir * q[c]);
    const double rho = pint[c + 1] / (rair * (tvp + tv) / 2.0);
    const double dpm = pm[c + 1] - pm[c];
    const double dc = bryan ? 0.0 : decay(c + 1);
    fm = g2dt * (bryan ? kmB[c + 1] : KmC * dc) * rho * rho / dpm;
    fe = g2dt * (bryan ? keB[c + 1] : KeC * dc) * rho * rho / dpm;
  };
  double ce = 0.0, cem = 0.0, cfu = 0.0, cfv = 0.0, cft = 0.0, cfq = 0.0;
  double fm_lo = 0.0, fe_lo = 0.0;   // the interface below level c
  for (int c = nz - 1; c >= 0; --c) {
    const double rp = 1.0 / (pint[c + 1] - pint[c]);
    double fm_up = 0.0, fe_up = 0.0;
    if (c > 0) iface(c - 1, fm_up, fe_up);
    // CAm / CCm, CA / CC of the reference: couplings to the level below / above
    const double am = (c < nz - 1) ? rp * fm_lo : 0.0, ae = (c < nz - 1) ? rp * fe_lo : 0.0;
    const double bm = (c > 0) ? rp * fm_up : 0.0, be = (c > 0) ? rp * fe_up : 0.0;
    const double de = 1.0 + ae + be - ae * ce, dmm = 1.0 + am + bm - am * cem;
    ce = be / de;
    cem = bm / dmm;
    cfu = (u[c] + am * cfu) / dmm;
    cfv = (v[c] + am * cfv) / dmm;
    cft = (pow(p0 / pm[c], kap) * t[c] + ae * cft) / de;
    cfq = (q[c] + ae * cfq) / de;
    CE[c] = ce; CEm[c] = cem; CFu[c] = cfu; CFv[c] = cfv; CFt[c] = cft; CFq[c] = cfq;
    fm_lo = fm_up;
    fe_lo = fe_up;
  }
  u[0] = CFu[0];
  v[0] = CFv[0];
  t[0] = CFt[0] * pow(pm[0] / p0, kap);
  q[0] = CFq[0];
  for (int c = 1; c < nz; ++c) {
    u[c] = CEm[c] * u[c - 1] + CFu[c];
    v[c] = CEm[c] * v[c - 1] + CFv[c];
    t[c] = (CE[c] * t[c - 1] * pow(p0 / pm[c - 1], kap) + CFt[c]) * pow(pm[c] / p0, kap);
    q[c] = CE[c] * q[c - 1] + CFq[c];
  }
  return precl;
}

// nhm/forcing/terminator.py:20-70 tendency_terminator at one level: the Cl
// tendency (Cl2's is minus half of it); sin, cos, exp and sqrt are CUDA's
__device__ __forceinline__ double terminator_cl_f(double lat_deg, double lon_deg, double cl, double cl2, double dt) {
  const double d2r = 3.141592653589793 / 180.0;
  const double lat_c = 20.0 * d2r, lon_c = 300.0 * d2r;
  const double la = lat_deg * d2r, lo = lon_deg * d2r;
  const double k1 = fmax(0.0, sin(la) * sin(lat_c) + cos(la) * cos(lat_c) * cos(lo - lon_c));
  const double k2 = 1.0;
  const double r = k1 / (4.0 * k2);
  const double cly = cl + 2.0 * cl2;
  const double det = sqrt(r * r + 2.0 * r * cly);
  const double expdt = exp(-4.0 * k2 * det * dt);
  const bool mask = fabs(det * k2 * dt) > 1.0e-16;
  const double el = mask ? (1.0 - expdt) / det / dt : 4.0 * k2;
  return -el * (cl - det + r) * (cl + det + r) / (1.0 + expdt + dt * el * (cl + r));
}

__global__ void k_forcing_dcmip(DcmipArgs a) {
  const int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l;
  if (!col_of(t, i, j, l)) return;
  const Col c = col_reg(i, j, l);
  const int KA = cD.KA, kmin = cD.kmin, kmax = cD.kmax, nz = kmax - kmin + 1;
  double* const* P = a.P.v;
  const double dt = a.dt;
  // diagnostics at level k (kernels/diag.py:53-143) with the water mixing ratios
  auto diag = [&](int k, double& rho, double& pre, double& tem, double& ein, double q[3]) {
    const int p = c.at(k);
    const double RHOG = P[0][p];
    rho = RHOG / cG.GSGAM2[p];
    ein = P[5][p] / RHOG;
    for (int n = 0; n < 3; ++n) q[n] = n < cC.nqw ? a.Pq[n][p] / RHOG : 0.0;   // DRY: vapour only
    double qd, cv;
    moist_qd_cv([&](int n) { return a.Pq[n][p] / RHOG; }, q[0], qd, cv);
    tem = ein / cv;
    pre = rho * tem * (qd * cC.Rdry + q[0] * cC.Rvap);
    if (a.negative_fixer)
      for (int n = 0; n < 3; ++n) q[n] = fmax(q[n], 0.0);
  };
  double th[NC_KESS_K], qv[NC_KESS_K], qc[NC_KESS_K], qr[NC_KESS_K], pk[NC_KESS_K];
  double prec = 0.0;
  if (a.kessler) {
  double r[NC_KESS_K], rh[NC_KESS_K], pc[NC_KESS_K], vq[NC_KESS_K], z[NC_KESS_K];
  // dry mixing ratios, dry density (in rh for now), Exner function, theta
  for (int m = 0; m < nz; ++m) {
    double rho, pre, tem, ein, q[3];
    diag(kmin + m, rho, pre, tem, ein, q);
    const double qd = 1.0 - q[0] - q[1] - q[2];
    qv[m] = q[0] / qd;
    qc[m] = q[1] / qd;
    qr[m] = q[2] / qd;
    rh[m] = rho * qd;
    pk[m] = pow(pre / a.PRE00, a.RdCp);
    th[m] = tem / pk[m];
    z[m] = a.zf[c.at(kmin + m)];
  }
  // kessler.py: constants, local arrays, CFL and sub-cycles
  const double f2x = 17.27, f5 = 237.3 * f2x * 2500000.0 / 1003.0, xk = 0.2875, psl = 1000.0, rhoqr = 1000.0;
  const double rho0 = rh[0];
  for (int m = 0; m < nz; ++m) {
    r[m] = 0.001 * rh[m];
    rh[m] = sqrt(rho0 / rh[m]);
    pc[m] = 3.8 / (pow(pk[m], 1.0 / xk) * psl);
    vq[m] = 36.34 * pow(qr[m] * r[m], 0.1364) * rh[m];
  }
  double cflmin = 0.0;
  for (int m = 0; m < nz - 1; ++m) {
    const double cfl = (vq[m] != 0.0) ? 0.8 * (z[m + 1] - z[m]) / vq[m] : dt;
    cflmin = (m == 0 || cfl < cflmin) ? cfl : cflmin;
  }
  const double dt_max = fmin(dt, cflmin);
  const int rainsplit = (int)ceil(dt / dt_max);
  const double dt0 = dt / (double)rainsplit;
  double precl = 0.0;
  for (int nt = 1; nt <= rainsplit; ++nt) {
    precl = precl + rho0 * qr[0] * vq[0] / rhoqr;
    // sedimentation from the start-of-sub-cycle rain (upstream), then the
    // level updates; sed of level m reads level m+1, so form it first
    double sed_next = 0.0;
    for (int m = 0; m < nz; ++m) {
      double sed;
      if (m < nz - 1) {
        const double num = r[m + 1] * qr[m + 1] * vq[m + 1] - r[m] * qr[m] * vq[m];
        sed = dt0 * num / (r[m] * (z[m + 1] - z[m]));
      } else {
        sed = -dt0 * qr[m] * vq[m] / (0.5 * (z[m] - z[m - 1]));
      }
      // level m - 1 is updated once level m's sedimentation (which reads its old rain) is formed
      if (m > 0) {
        const int u = m - 1;
        const double qc0 = qc[u], qr0 = qr[u], qv0 = qv[u], th0 = th[u];
        const double qrprod = qc0 - (qc0 - dt0 * fmax(0.001 * (qc0 - 0.001), 0.0)) / (1.0 + dt0 * 2.2 * pow(qr0, 0.875));
        const double qc1 = fmax(qc0 - qrprod, 0.0);
        const double qr1 = fmax(qr0 + qrprod + sed_next, 0.0);
        const double pkt = pk[u] * th0;
        const double qvs = pc[u] * exp(f2x * (pkt - 273.0) / (pkt - 36.0));
        const double prod = (qv0 - qvs) / (1.0 + qvs * f5 / ((pkt - 36.0) * (pkt - 36.0)));
        const double rqr = r[u] * qr1;
        const double ern =
            fmin(fmin(dt0 * (((1.6 + 124.9 * pow(rqr, 0.2046)) * pow(rqr, 0.525)) /
                             (2550000.0 * pc[u] / (3.8 * qvs) + 540000.0)) *
                          (fmax(qvs - qv0, 0.0) / (r[u] * qvs)),
                      fmax(-prod - qc1, 0.0)),
                 qr1);
        const double mpc = fmax(prod, -qc1);
        th[u] = th0 + 2500000.0 / (1003.0 * pk[u]) * (mpc - ern);
        qv[u] = fmax(qv0 - mpc + ern, 0.0);
        qc[u] = qc1 + mpc;
        qr[u] = qr1 - ern;
      }
      sed_next = sed;
    }
    {   // the top level
      const int u = nz - 1;
      const double qc0 = qc[u], qr0 = qr[u], qv0 = qv[u], th0 = th[u];
      const double qrprod = qc0 - (qc0 - dt0 * fmax(0.001 * (qc0 - 0.001), 0.0)) / (1.0 + dt0 * 2.2 * pow(qr0, 0.875));
      const double qc1 = fmax(qc0 - qrprod, 0.0);
      const double qr1 = fmax(qr0 + qrprod + sed_next, 0.0);
      const double pkt = pk[u] * th0;
      const double qvs = pc[u] * exp(f2x * (pkt - 273.0) / (pkt - 36.0));
      const double prod = (qv0 - qvs) / (1.0 + qvs * f5 / ((pkt - 36.0) * (pkt - 36.0)));
      const double rqr = r[u] * qr1;
      const double ern =
          fmin(fmin(dt0 * (((1.6 + 124.9 * pow(rqr, 0.2046)) * pow(rqr, 0.525)) /
                           (2550000.0 * pc[u] / (3.8 * qvs) + 540000.0)) *
                        (fmax(qvs - qv0, 0.0) / (r[u] * qvs)),
                    fmax(-prod - qc1, 0.0)),
               qr1);
      const double mpc = fmax(prod, -qc1);
      th[u] = th0 + 2500000.0 / (1003.0 * pk[u]) * (mpc - ern);
      qv[u] = fmax(qv0 - mpc + ern, 0.0);
      qc[u] = qc1 + mpc;
      qr[u] = qr1 - ern;
    }
    if (nt < rainsplit)
      for (int m = 0; m < nz; ++m) vq[m] = 36.34 * pow(qr[m] * r[m], 0.1364) * rh[m];
  }
  prec = prec + precl / (double)rainsplit;
  }   // Kessler
  // simple physics from the same state, top down (mod_af_dcmip.py:230-317)
  double st[NC_KESS_K], sq[NC_KESS_K], su[NC_KESS_K], sv[NC_KESS_K];
  const int cidx = (l * cD.G + j) * cD.G + i;
  const int npl = cD.L * cD.G * cD.G;
  if (a.sm) {
    double pm[NC_KESS_K], pint[NC_KESS_K + 1];
    double w1[NC_KESS_K], w2[NC_KESS_K], w3[NC_KESS_K], w4[NC_KESS_K], w5[NC_KESS_K], w6[NC_KESS_K];
    const double* IJ = a.ij;
    double alt_up = 0.0, alth_up = 0.0;
    for (int cc = 0; cc < nz; ++cc) {
      const int k = kmax - cc, p = c.at(k);
      double rho, pre, tem, ein, q[3];
      diag(k, rho, pre, tem, ein, q);
      const double RHOG = P[0][p];
      const double vx = P[1][p] / RHOG, vy = P[2][p] / RHOG, vz = P[3][p] / RHOG;
      st[cc] = tem;
      sq[cc] = q[0];
      su[cc] = vx * IJ[cidx] + vy * IJ[npl + cidx] + vz * IJ[2 * npl + cidx];
      sv[cc] = vx * IJ[3 * npl + cidx] + vy * IJ[4 * npl + cidx] + vz * IJ[5 * npl + cidx];
      pm[cc] = pre;
      const double alt = a.zf[p], alth = a.zh[p];
      if (cc > 0)   // log-interpolated interface pressure (mod_af_dcmip.py:254-259)
        pint[cc] = pm[cc] * exp(log(pm[cc - 1] / pm[cc]) * (alth_up - alt) / (alt_up - alt));
      alt_up = alt;
      alth_up = alth;
    }
    double ps;
    {   // single-layer hydrostatic surface pressure (mod_forcing.py:250)
      double rho, pre, tem, ein, q[3];
      diag(kmin, rho, pre, tem, ein, q);
      ps = pre + rho * cC.GRAV * (a.zf[c.at(kmin)] - a.zsfc[cidx]);
    }
    pint[0] = 0.0;
    pint[nz] = ps;
    prec = prec + simple_physics_col(nz, st, sq, su, sv, pm, pint, ps, a.tsurf[cidx], dt, a.sm_lsc, a.sm_C,
                                     a.sm_bryan, w1, w2, w3, w4, w5, w6);
  }
  double hs_psref = 0.0, sin2 = 0.0, cos2 = 0.0, cos4 = 0.0;
  if (a.hs) {   // moist Held-Suarez: the reference surface pressure of the column
    double rho, pre, tem, ein, q[3];
    diag(kmin, rho, pre, tem, ein, q);
    const double pre_kmin = pre;
    diag(kmin - 1, rho, pre, tem, ein, q);
    hs_psref = 0.5 * (pre_kmin + pre);
    sin2 = a.hs_lat3[cidx];
    cos2 = a.hs_lat3[npl + cidx];
    cos4 = a.hs_lat3[2 * npl + cidx];
  }
  a.precip[cidx] = prec;
  // back to wet mixing ratios, the tendencies, and their application on every level
  for (int k = 0; k < KA; ++k) {
    const int p = c.at(k);
    double rho, pre, tem, ein, q[3];
    diag(k, rho, pre, tem, ein, q);
    double fe = 0.0, fq[3] = {0.0, 0.0, 0.0}, fv[3] = {0.0, 0.0, 0.0}, fcl = 0.0, fcl2 = 0.0;
    if (k >= kmin && k <= kmax && a.n_cl >= 0) {   // mod_af_dcmip.py:171-187
      const double d2r = 3.141592653589793 / 180.0;
      const double lat_deg = a.lat[cidx] / d2r, lon_deg = a.lon[cidx] / d2r;
      const double RHOG = P[0][p];
      double qcl = a.Pq[a.n_cl][p] / RHOG, qcl2 = a.Pq[a.n_cl2][p] / RHOG;
      if (a.negative_fixer) {
        qcl = fmax(qcl, 0.0);
        qcl2 = fmax(qcl2, 0.0);
      }
      const double qvd = 1.0 - q[0];
      const double cl_f = terminator_cl_f(lat_deg, lon_deg, qcl / qvd, qcl2 / qvd, dt);
      fcl = cl_f * qvd;
      fcl2 = (-cl_f / 2.0) * qvd;
    }
    if (k >= kmin && k <= kmax && a.kessler) {
      const int m = k - kmin;
      const double qd2 = 1.0 / (1.0 + qv[m] + qc[m] + qr[m]);
      const double qvk = qv[m] * qd2, qck = qc[m] * qd2, qrk = qr[m] * qd2;
      const double cvk = qd2 * cC.CVdry + qvk * cC.CVW[0] + qck * cC.CVW[1] + qrk * cC.CVW[2];
      fq[0] = fq[0] + (qvk - q[0]) / dt;
      fq[1] = fq[1] + (qck - q[1]) / dt;
      fq[2] = fq[2] + (qrk - q[2]) / dt;
      const double tem_new = th[m] * pk[m];
      const double cv_old = ein / tem;
      const double dtem = tem_new - tem;
      const double dcv = cvk - cv_old;
      fe = fe + (cv_old * dtem + tem * dcv + dcv * dtem) / dt;
    }
    if (k >= kmin && k <= kmax && a.sm) {   // mod_af_dcmip.py:472-511 (DRY or WARM)
      const int cc = kmax - k;
      const double RHOG = P[0][p];
      const double vel[3] = {P[1][p] / RHOG, P[2][p] / RHOG, P[3][p] / RHOG};
      for (int d = 0; d < 3; ++d)
        fv[d] = (su[cc] * a.ij[d * npl + cidx] + sv[cc] * a.ij[(3 + d) * npl + cidx] - vel[d]) / dt;
      const double qvn = sq[cc];
      double cv;
      if (cC.nqw == 3) {
        const double qd = 1.0 - qvn - q[1] - q[2];
        cv = qd * cC.CVdry + qvn * cC.CVW[0] + q[1] * cC.CVW[1] + q[2] * cC.CVW[2];
      } else {   // RAIN_TYPE DRY
        const double qd = 1.0 - qvn;
        cv = qd * cC.CVdry + qvn * cC.CVW[0];
      }
      fq[0] = fq[0] + (qvn - q[0]) / dt;
      const double cv_old = ein / tem;
      const double dtem = st[cc] - tem;
      const double dcv = cv - cv_old;
      fe = fe + (cv_old * dtem + tem * dcv + dcv * dtem) / dt;
    }
    if (k >= kmin && k <= kmax && a.hs) {   // mod_forcing.py:278-287: HS momentum replaces, HS energy adds
      const double RHOG = P[0][p];
      double hfe;
      hs_tendency(a.hp, sin2, cos2, cos4, hs_psref, pre, tem, P[1][p] / RHOG, P[2][p] / RHOG, P[3][p] / RHOG, fv[0],
                  fv[1], fv[2], hfe);
      fe = fe + hfe;
    }
    const double gs = cG.GSGAM2[p];
    P[1][p] = P[1][p] + dt * fv[0] * rho * gs;
    P[2][p] = P[2][p] + dt * fv[1] * rho * gs;
    P[3][p] = P[3][p] + dt * fv[2] * rho * gs;
    P[5][p] = P[5][p] + dt * fe * rho * gs;
    double rhog = P[0][p];
    for (int n = 0; n < a.nq; ++n) {
      const double f = n < cC.nqw ? fq[n] : (n == a.n_cl ? fcl : (n == a.n_cl2 ? fcl2 : 0.0));
      double frhogq = f * rho * gs;
      double* Q = a.Pq[n];
      if (a.negative_fixer) {
        const double tmp = fmax(Q[p] + dt * frhogq, 0.0);
        frhogq = (tmp - Q[p]) / dt;
        Q[p] = tmp;
      } else {
        Q[p] = Q[p] + dt * frhogq;
      }
      if (a.update_tot_dens && n < cC.nqw) rhog = rhog + dt * frhogq;
    }
    P[0][p] = rhog;
  }
}

}  // namespace nc

namespace nc {

// ---------------------------------------------------------------------------
// Offline tracer advection (integ_type TRCADV): the prescribed winds of
// DCMIP2012 test 1-1 set after each step (nhm/forcing/mod_forcing.py
// forcing_update; nhm/forcing/mod_af_trcadv.py test11_velocity,
// Sp_Unit_East / Sp_Unit_North).  exp, sin and cos are CUDA's, so the winds
// can differ from numpy's in the last bits.
// ---------------------------------------------------------------------------
template <class R>
struct TrcWindArgs {
  Prog<R> P;                  // RHOGV{X,Y,Z}, RHOGW set to wind * RHOG (float64 arithmetic in both forms)
  const double *lon, *lat;    // column longitude / latitude: regional [l][j][i], pole [g][l]
  const double *zf, *zh;      // full / half-level height: regional [l][k][j][i], pole [g][k][l]
  const double* time;         // model time of the winds (device scalar)
  double a, Rd, g, pi;        // the test's constants (mod_af_trcadv.py:14-19)
  int hadley;                 // DCMIP 1-2 (test12_velocity) instead of 1-1
};

// DCMIP2012 test 1-2, Hadley-like meridional circulation (nhm/forcing/
// mod_af_trcadv.py:100-149 test12_velocity): the full-level winds (u, v) and
// the half-level w at one point
__device__ __forceinline__ void trcadv12(double time, double lat, double zf, double zh, double a, double Rd, double g,
                                         double pi, double& u, double& v, double& ww) {
  const double tau = 1.0 * 86400.0, u0 = 40.0, w0 = 0.15, T0 = 300.0;
  const double H = Rd * T0 / g;
  const double K = 5.0, ztop = 12.0e3, p0 = 1000.e2;
  const double rho0 = p0 / (Rd * T0);
  double rho = p0 * exp(-zf / H) / (Rd * T0);
  u = u0 * cos(lat);
  v = -(rho0 / rho) * a * w0 * pi / (K * ztop) * cos(lat) * sin(K * lat) * cos(pi * zf / ztop) * cos(pi * time / tau);
  rho = p0 * exp(-zh / H) / (Rd * T0);
  ww = (rho0 / rho) * (w0 / K) * (-2.0 * sin(K * lat) * sin(lat) + K * cos(lat) * cos(K * lat)) *
       sin(pi * zh / ztop) * cos(pi * time / tau);
}

__global__ void k_trcadv_time(double* time, double dt) { *time = *time + dt; }

// one thread per point of the regional (pole == 0) or pole (pole != 0) grid
template <class R>
__global__ void k_trcadv_winds(TrcWindArgs<R> w, int pole) {
  const int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  const int KA = cD.KA;
  int p, c2;   // point index and column index of lon/lat
  if (!pole) {
    if (t >= cD.npti) return;
    const int G = cD.G;
    const int i = t % G, j = (t / G) % G, l = t / (G * G * KA);
    p = t;
    c2 = (l * G + j) * G + i;
  } else {
    if (t >= 6 * KA * cD.LP) return;
    const int g = t / (KA * cD.LP), lp = t % cD.LP;
    p = t;
    c2 = g * cD.LP + lp;
  }
  const double time = *w.time;
  const double a = w.a, pi = w.pi;
  if (w.hadley) {
    const double lon = w.lon[c2], lat = w.lat[c2];
    double u, v, ww;
    trcadv12(time, lat, w.zf[p], w.zh[p], a, w.Rd, w.g, pi, u, v, ww);
    const double e0 = -sin(lon), e1 = cos(lon), e2 = 0.0;
    const double n0 = -sin(lat) * cos(lon), n1 = -sin(lat) * sin(lon), n2 = cos(lat);
    const double vx = e0 * u + n0 * v, vy = e1 * u + n1 * v, vz = e2 * u + n2 * v;
    const double rg = (double)w.P.v[0][p];
    w.P.v[1][p] = vx * rg;
    w.P.v[2][p] = vy * rg;
    w.P.v[3][p] = vz * rg;
    w.P.v[4][p] = ww * rg;
    return;
  }
  const double tau = 12.0 * 86400.0;
  const double u0 = 2.0 * pi * a / tau;
  const double k0 = 10.0 * a / tau;
  const double omega0 = 23000.0 * pi / tau;
  const double T0 = 300.0;
  const double H = w.Rd * T0 / w.g;
  const double p0 = 1000.E2;
  const double dlon = 2.0 * pi * time / tau;
  const double lon = w.lon[c2], lat = w.lat[c2];
  const double lonp = lon - dlon;
  const double bs = 0.2;
  const double ptop = p0 * exp(-12000.0 / H);
  // full level
  double pf = p0 * exp(-w.zf[p] / H);
  const double cl = cos(lat);
  const double ud = (omega0 * a) / (bs * ptop) * cos(lonp) * (cl * cl) * cos(dlon) *
                    (-exp((pf - p0) / (bs * ptop)) + exp((ptop - pf) / (bs * ptop)));
  const double sl = sin(lonp);
  const double u = k0 * sin(2.0 * lat) * (sl * sl) * cos(0.5 * dlon) + u0 * cl + ud;
  const double v = k0 * sin(2.0 * lonp) * cl * cos(0.5 * dlon);
  const double e0 = -sin(lon), e1 = cos(lon), e2 = 0.0;
  const double n0 = -sin(lat) * cos(lon), n1 = -sin(lat) * sin(lon), n2 = cl;
  const double vx = e0 * u + n0 * v, vy = e1 * u + n1 * v, vz = e2 * u + n2 * v;
  // half level
  const double ph = p0 * exp(-w.zh[p] / H);
  const double s = (1.0 + exp((ptop - p0) / (bs * ptop)) - exp((ph - p0) / (bs * ptop)) -
                    exp((ptop - ph) / (bs * ptop)));
  const double ww = -(w.Rd * T0) / (w.g * ph) * omega0 * sl * cl * cos(dlon) * s;
  const double rg = (double)w.P.v[0][p];
  w.P.v[1][p] = vx * rg;
  w.P.v[2][p] = vy * rg;
  w.P.v[3][p] = vz * rg;
  w.P.v[4][p] = ww * rg;
}

}  // namespace nc
