// Artificial forcing after the dynamics step (Dyn.forcing_step,
// pynicamdc/nhm/dynamics/mod_dynamics.py:597-735): the Held-Suarez case.
#pragma once
#include "nc_small.cuh"

namespace nc {

// Held & Suarez (1994) dry-case parameters (nhm/forcing/mod_af_heldsuarez.py:19-36)
struct HsArgs {
  Prog P;                 // PROG, updated in place
  const double* Pq0;      // first tracer (water vapour) for the diagnostics
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
    const double q0 = a.Pq0[p] / RHOG;
    const double qd = 1.0 - q0;
    const double cv = q0 * cC.CVW0 + qd * cC.CVdry;
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
