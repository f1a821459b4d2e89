// Artificial forcing after the dynamics step (Dyn.forcing_step,
// pynicamdc/nhm/dynamics/mod_dynamics.py:597-735): the Held-Suarez case.
#pragma once
#include "nc_small.cuh"

namespace nc {

// Held & Suarez (1994) dry-case parameters (nhm/forcing/mod_af_heldsuarez.py:19-36)
struct HsArgs {
  Prog<double> P;         // PROG, updated in place
  const double* Pqw[NC_MAXQW];   // the water tracers (0: vapour) for the diagnostics
  const double* lat3;     // planes |sin lat|^2, |cos lat|^2, |cos lat|^4 of each column
  double dt, RdCp;        // large time step; Rdry / CPdry
  double sigma_b, Kf, Dth_z, Ka, Ks, T_eq0, DT_y, PRE00;
};

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
    const double sigma = pre / psref;
    const double factor = npmax((sigma - a.sigma_b) / (1.0 - a.sigma_b), 0.0);
    const double fvx = -a.Kf * factor * vx;
    const double fvy = -a.Kf * factor * vy;
    const double fvz = -a.Kf * factor * vz;
    const double ap0 = fabs(pre / a.PRE00);
    const double Kt = a.Ka + (a.Ks - a.Ka) * factor * cos4;
    const double T_eq = npmax(200.0, (a.T_eq0 - a.DT_y * sin2 - a.Dth_z * log(npmax(ap0, 1e-30)) * cos2) *
                                         pow(ap0, a.RdCp));
    const double fe = -Kt * (tem - T_eq) * cC.CVdry;
    const double gs = cG.GSGAM2[p];
    P[0][p] = P[0][p] + 0.0;
    P[1][p] = P[1][p] + a.dt * fvx * rho * gs;
    P[2][p] = P[2][p] + a.dt * fvy * rho * gs;
    P[3][p] = P[3][p] + a.dt * fvz * rho * gs;
    P[4][p] = P[4][p] + 0.0;
    P[5][p] = P[5][p] + a.dt * fe * rho * gs;
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
};

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
