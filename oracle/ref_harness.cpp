// ref_harness.cpp -- extern "C" entry points into the reference AAK code,
// compiled together with the UNMODIFIED reference sources (read in place from
// the reference checkout by oracle/Makefile) into oracle/_ref/libaakref.so.
//
// Test infrastructure only: the parity tests and the CPU-baseline leg of the
// benchmark load this library to run the reference itself.  The product
// library never links it.
//
// The glue below repeats the reference's own call sequences so that the
// individual stages can be observed:
//   ref_front      : src/suite/AAKpy.cc:20-44   (GKTrajFast + Frequencies + ParAng + ParMap)
//   ref_genwave    : src/suite/AAK.cc:565-591   (GenWave packing) with an optional nmodes override
//   ref_aakwave    : src/suite/AAKpy.cc:16-51   (AAKwave itself)
//   ref_aakphase   : src/suite/AAKpy.cc:53-88   (AAKphase itself)
//   ref_genphase   : src/suite/AAKPhase.cc:315-374 (GenPhase on a mapped trajectory)
//   ref_aaktdi     : src/suite/AAKpy.cc:90-125  (AAKTDI itself)
//   ref_gentdi     : src/suite/AAKTDI.cc:799-829 (GenTDI on a mapped trajectory)
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <vector>

#include "Globals.h"
#include "GKTrajFast.h"
#include "KSParMap.h"
#include "KSTools.h"
#include "AAK.h"
#include "AAKpy.h"
#include "IEKG.h"
#include "GKR.h"
#include "CKG.h"
#include "AAKPhase.h"
#include "AAKTDI.h"
#include "AKTDI.h"

// The reference's AAKpy.cc also defines AKTDI, whose callee lives in a
// translation unit outside this build.  It is never called through this
// harness; this definition only satisfies the linker.
void GenAKTDI(double *, double *, double *, double *, double *, double *, double *, double, int, double, double,
              double, double, double, double, double, double, double, double, double, double, double, double,
              bool, bool) {
  std::abort();
}

extern "C" {

// Flat parameter record, the numeric fields of SetPar (include/KSTools.h:21-53).
struct ref_params {
  double length, dt, p, T, f, T_fit, mu, M, s, e, iota, gamma, psi, theta_S, phi_S, theta_K, phi_K, alpha, D;
  int backint, LISA;
};

static void to_setpar(const ref_params *r, SetPar *s) {
  std::memset(s, 0, sizeof(SetPar));
  std::strcpy(s->path, "oracle");
  s->backint = r->backint != 0;
  s->LISA = r->LISA != 0;
  s->traj = false;
  s->SNR = false;
  s->timing = false;
  s->length = (int)r->length;
  s->dt = r->dt;
  s->p = r->p;
  s->T = r->T;
  s->f = r->f;
  s->T_fit = r->T_fit;
  s->mu = r->mu;
  s->M = r->M;
  s->s = r->s;
  s->e = r->e;
  s->iota = r->iota;
  s->gamma = r->gamma;
  s->psi = r->psi;
  s->theta_S = r->theta_S;
  s->phi_S = r->phi_S;
  s->theta_K = r->theta_K;
  s->phi_K = r->phi_K;
  s->alpha = r->alpha;
  s->D = r->D;
}

double ref_aakwave(const ref_params *r, double *t, double *hI, double *hII) {
  SetPar s;
  to_setpar(r, &s);
  return AAKwave(s, t, hI, hII);
}

double ref_aakphase(const ref_params *r, double *t, double *phase_r, double *phase_theta, double *phase_phi,
                    double *omega_r, double *omega_theta, double *omega_phi, double *eccentricity) {
  SetPar s;
  to_setpar(r, &s);
  return AAKphase(s, t, phase_r, phase_theta, phase_phi, omega_r, omega_theta, omega_phi, eccentricity);
}

double ref_aaktdi(const ref_params *r, double *f, double *Xr, double *Xi, double *Yr, double *Yi, double *Zr,
                  double *Zi) {
  SetPar s;
  to_setpar(r, &s);
  return AAKTDI(s, f, Xr, Xi, Yr, Yi, Zr, Zi);
}

// GenTDI (AAKTDI.cc:799-829) on a mapped trajectory; outputs hold (vlength + 1) / 2 entries.
void ref_gentdi(double *f, double *Xr, double *Xi, double *Yr, double *Yi, double *Zr, double *Zi, double timestep,
                int vlength, const double *e_traj, const double *v_map, double M_phys, const double *M_map,
                double mu, double S_phys, const double *S_map, double dist, double inc, double gim0, double Phi0,
                double qS, double phiS, double alp0, double qK, double phiK, const double *dt_map, int steps,
                int backint) {
  GenTDI(f, Xr, Xi, Yr, Yi, Zr, Zi, timestep, vlength, (double *)e_traj, (double *)v_map, M_phys, (double *)M_map,
         mu, S_phys, (double *)S_map, dist, inc, gim0, Phi0, qS, phiS, alp0, qK, phiK, (double *)dt_map, steps,
         backint != 0, false, false);
}

// GenPhase (AAKPhase.cc:315-374) on a mapped trajectory; outputs hold vlength entries.
void ref_genphase(double *t, double *phase_r, double *phase_theta, double *phase_phi, double *omega_r,
                  double *omega_theta, double *omega_phi, double *eccentricity, double timestep, int vlength,
                  const double *e_traj, const double *v_map, double M_phys, const double *M_map, double mu,
                  double S_phys, const double *S_map, double dist, double inc, double gim0, double Phi0, double qS,
                  double phiS, double alp0, double qK, double phiK, const double *dt_map, int steps, int backint) {
  GenPhase(t, phase_r, phase_theta, phase_phi, omega_r, omega_theta, omega_phi, eccentricity, timestep, vlength,
           (double *)e_traj, (double *)v_map, M_phys, (double *)M_map, mu, S_phys, (double *)S_map, dist, inc, gim0,
           Phi0, qS, phiS, alp0, qK, phiK, (double *)dt_map, steps, backint != 0, false, false);
}

// Front end of AAKwave: coarse Kerr inspiral, Kerr frequencies, initial mean
// anomaly and the Kerr->AK parameter map.  Arrays must hold >= 100 entries.
// traj_out (optional) receives per step: t[RR], p, e, cosiota, E, Lz, Q, Omega_r, Omega_theta, Omega_phi.
int ref_front(const ref_params *r, int *steps_out, double *e_traj, double *v_map, double *M_map,
              double *s_map, double *dt_map, double *Phi0_out, double *traj_out) {
  SetPar A;
  to_setpar(r, &A);
  GKTrajFast gktraj3(cos(A.iota), A.s);
  gktraj3.p = A.p;
  gktraj3.ecc = A.e;
  int maxsteps = 100;
  int steps = 0;
  double dt_fit = std::min(A.T_fit, A.length * A.dt / SOLARMASSINSEC / A.M / A.M * A.mu) / (maxsteps - 1);
  TrajData *traj3 = (TrajData *)malloc((size_t)((maxsteps + 1) * sizeof(TrajData)));
  int flag = gktraj3.Eccentric(dt_fit, traj3, maxsteps, steps);
  double Omega_t[3], ang[3], map_t[3];
  double Phi = 0.0;
  for (int i = 1; i <= steps; i++) {
    IEKG geodesic_t(traj3[i].p, traj3[i].ecc, traj3[i].cosiota, A.s);
    geodesic_t.Frequencies(Omega_t);
    if (i == 1) {
      ParAng(ang, A.e, A.iota, A.gamma, A.psi, A.theta_S, A.phi_S, A.theta_K, A.phi_K, A.alpha,
             geodesic_t.zedminus);
      Phi = ang[0];
    }
    ParMap(map_t, Omega_t, traj3[i].p, A.M, A.s, traj3[i].ecc, A.iota);
    e_traj[i - 1] = traj3[i].ecc;
    v_map[i - 1] = map_t[0];
    M_map[i - 1] = map_t[1];
    s_map[i - 1] = map_t[2];
    dt_map[i - 1] = traj3[i].t * SOLARMASSINSEC * A.M * A.M / A.mu;
    if (traj_out) {
      double *o = traj_out + 10 * (i - 1);
      o[0] = traj3[i].t;
      o[1] = traj3[i].p;
      o[2] = traj3[i].ecc;
      o[3] = traj3[i].cosiota;
      o[4] = traj3[i].E;
      o[5] = traj3[i].Lz;
      o[6] = traj3[i].Q;
      o[7] = Omega_t[0];
      o[8] = Omega_t[1];
      o[9] = Omega_t[2];
    }
  }
  free(traj3);
  *steps_out = steps;
  *Phi0_out = Phi;
  return flag;
}

// GenWave packing (AAK.cc:565-591) followed by waveform(); nmodes_override <= 0
// keeps the reference rule int(30 e0) / 4.
void ref_genwave(double *t, double *hI, double *hII, double timestep, int vlength, const double *e_traj,
                 const double *v_map, double M_phys, const double *M_map, double mu, double S_phys,
                 const double *S_map, double dist, double inc, double gim0, double Phi0, double qS, double phiS,
                 double alp0, double qK, double phiK, const double *dt_map, int steps, int backint, int mich,
                 int nmodes_override) {
  double par[12];
  par[0] = mu * SOLARMASSINSEC;
  par[1] = M_map[0] * SOLARMASSINSEC;
  par[2] = S_map[0];
  par[3] = e_traj[0];
  par[4] = inc;
  par[5] = gim0;
  par[6] = Phi0;
  par[7] = qS;
  par[8] = phiS;
  par[9] = qK;
  par[10] = phiK;
  par[11] = alp0;
  int nmodes = (int)(30 * par[3]);
  if (par[3] < 0.135) nmodes = 4;
  if (nmodes_override > 0) nmodes = nmodes_override;
  double zeta = par[0] / dist / Gpc;
  // waveform() writes t/hI/hII[0..vlength-1]
  waveform(t, hI, hII, timestep, vlength, nmodes, zeta, par, (double *)e_traj, (double *)v_map, M_phys,
           (double *)M_map, S_phys, (double *)S_map, (double *)dt_map, steps, backint != 0, mich != 0, false);
}

// PNevolution (AAK.cc:27-318) with the GenWave packing; dense arrays have vlength+1 entries.
void ref_pnevolution(double timestep, int vlength, const double *e_traj, const double *v_map, double M_phys,
                     const double *M_map, double mu, double S_phys, const double *S_map, double inc, double gim0,
                     double Phi0, double alp0, const double *dt_map, int steps, int backint, double *t, double *e,
                     double *v, double *M, double *S, double *gim, double *Phi, double *alp, double *nu,
                     double *gimdot, int *i_plunge, int *i_buffer) {
  double par[12] = {0};
  par[0] = mu * SOLARMASSINSEC;
  par[1] = M_map[0] * SOLARMASSINSEC;
  par[2] = S_map[0];
  par[3] = e_traj[0];
  par[4] = inc;
  par[5] = gim0;
  par[6] = Phi0;
  par[11] = alp0;
  PNevolution(t, e, v, M, S, gim, Phi, alp, nu, gimdot, timestep, vlength, par, (double *)e_traj,
              (double *)v_map, M_phys, (double *)M_map, S_phys, (double *)S_map, (double *)dt_map, steps,
              i_plunge, i_buffer, backint != 0);
}

// IEKG (src/inclecc/IEKG.cc): out = E, Lz, Q, Stable, r1, r2, r3, r4, zedminus, zedplus,
// Omega_r, Omega_theta, Omega_phi (the frequencies only when Stable == 1).
void ref_iekg(double p, double e, double cosi, double a, double *out) {
  IEKG g(p, e, cosi, a);
  out[0] = g.E;
  out[1] = g.Lz;
  out[2] = g.Q;
  out[3] = g.Stable;
  out[4] = g.r1;
  out[5] = g.r2;
  out[6] = g.r3;
  out[7] = g.r4;
  out[8] = g.zedminus;
  out[9] = g.zedplus;
  double Om[3] = {NAN, NAN, NAN};
  if (g.Stable == 1) g.Frequencies(Om);
  out[10] = Om[0];
  out[11] = Om[1];
  out[12] = Om[2];
}

// GKR fluxes (src/inclecc/GKR.cc:28-97) at (p, e, cosiota) using IEKG constants.
void ref_gkr(double p, double e, double cosi, double a, double *out) {
  IEKG g(p, e, cosi, a);
  GKR k(p, e, g.E, g.Lz, g.Q, a);
  out[0] = k.pdot;
  out[1] = k.edot;
  out[2] = k.cosidot;
  out[3] = k.Edot;
  out[4] = k.Lzdot;
  out[5] = k.Qdot;
}

// CKG circular constants (src/circ/CKG.cc:63-128), flag USING_cosiota.
void ref_ckg(double r, double cosi, double a, double *out) {
  CKG c(0, 0, cosi, USING_cosiota, r, a);
  out[0] = c.E;
  out[1] = c.Lz;
  out[2] = c.Q;
  out[3] = c.Lovercosi;
}

// LSO table of GKTrajFast's constructor (GKTrajFast.cc:20-130) and P_lso.
void ref_plso(double cosi, double a, int n, const double *csi, const double *e, double *out) {
  GKTrajFast g(cosi, a);
  for (int k = 0; k < n; ++k) out[k] = g.P_lso(csi[k], e[k]);
}
void ref_lso_table(double cosi, double a, double *out4) {
  GKTrajFast g(cosi, a);
  out4[0] = g.p_lso[1][1];
  out4[1] = g.p_lso[1][2];
  out4[2] = g.p_lso[2][1];
  out4[3] = g.p_lso[2][2];
}

void ref_parmap(double *map, const double *Omega, double p, double M, double s, double e, double iota) {
  ParMap(map, (double *)Omega, p, M, s, e, iota);
}
void ref_parang(double *ang, double e, double iota, double gamma, double psi, double theta_S, double phi_S,
                double theta_K, double phi_K, double alpha, double zm) {
  ParAng(ang, e, iota, gamma, psi, theta_S, phi_S, theta_K, phi_K, alpha, zm);
}
void ref_rotcoeff(double *rot, double iota, double theta_S, double phi_S, double theta_K, double phi_K,
                  double alpha) {
  RotCoeff(rot, iota, theta_S, phi_S, theta_K, phi_K, alpha);
}
void ref_pn_rates(double v, double e, double Y, double q, double m, double M, double *out) {
  out[0] = dtdm(v, e, Y, q);
  out[1] = drdm(v, e, Y, q);
  out[2] = dthetadm(v, e, Y, q);
  out[3] = dphidm(v, e, Y, q);
  out[4] = dvdt(v, e, Y, m, M, q);
  out[5] = dedt(v, e, Y, m, M, q);
}
void ref_polyfit(double *coeff, const double *x, const double *y, int n) {
  PolyFit(coeff, (double *)x, (double *)y, n);
}
void ref_interp(const double *x_in, const double *y_in, int n_in, const double *x_out, double *y_out, int n_out) {
  Interp((double *)x_in, (double *)y_in, n_in, (double *)x_out, y_out, n_out);
}
double ref_elisa_noise(double f) { return eLISA_Noise(f); }

}  // extern "C"
