// nb_step.cu -- the RESPA step on the device.
//
// Restates step() (integrate/md_step.c:62-159) for NVE with the level
// structure ninter (nres_lrf) / ninrra (nres_tors) / ninnra (nres_intra), the
// force levels of force() (energy/control/md_fcntr.c:44-134), nrefsh()
// (energy/control/md_finter.c:43-108, with its RESETPOS pull-back) and the
// harmonic fbond/fbend of the inner level (energy/intra/md_fbond.c:76-125,
// md_fbend.c:126-260).
//
// Bonds, bends and excluded-pair corrections only couple atoms of one
// molecule, so the atoms are partitioned into groups (connected components
// of those terms) and one thread owns a group: the whole inner loop -- every
// ninnra substep with its bonded forces -- runs in one kernel with no grid
// synchronisation, followed by the displacement test of nrefsh.  The
// excluded-pair correction (ecorr) and the bonded energies of getvireal are
// likewise per-group.
#include <math.h>

#include <algorithm>
#include <numeric>

#include "nb_common.cuh"

namespace cm3d {

struct StepP {
  int n, ngroups, ninrra, ninnra;
  double dter, dter1, dts2, dtr2, dta2;
  double skin2q;      // (skin/2)^2 = .25 skin^2  (md_finter.c:63)
  double kappa, kappa2;
  int use_fxs;
};

// bonded forces of one group into fxa (raw forces), fbond/fbend in CM3D's order
__device__ __forceinline__ void group_bonded(int g, int n, const double *__restrict__ pos,
                                             double *__restrict__ fxa, const int *__restrict__ gboff,
                                             const int4 *__restrict__ bij, const double2 *__restrict__ bp,
                                             const int *__restrict__ geoff, const int4 *__restrict__ eijk,
                                             const double2 *__restrict__ ep) {
  for (int b = gboff[g]; b < gboff[g + 1]; b++) {
    const int i = bij[b].x, j = bij[b].y;
    double dx = pos[i] - pos[j], dy = pos[n + i] - pos[n + j], dz = pos[2 * n + i] - pos[2 * n + j];
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    double dr = r - bp[b].x;
    double fr = bp[b].y * dr / r;
    dx *= fr; dy *= fr; dz *= fr;
    fxa[i] -= dx; fxa[n + i] -= dy; fxa[2 * n + i] -= dz;
    fxa[j] += dx; fxa[n + j] += dy; fxa[2 * n + j] += dz;
  }
  for (int b = geoff[g]; b < geoff[g + 1]; b++) {
    const int i = eijk[b].x, j = eijk[b].y, k = eijk[b].z;
    double ax = pos[i] - pos[j], ay = pos[n + i] - pos[n + j], az = pos[2 * n + i] - pos[2 * n + j];
    double al = ax * ax + ay * ay + az * az;
    double bx = pos[k] - pos[j], by = pos[n + k] - pos[n + j], bz = pos[2 * n + k] - pos[2 * n + j];
    double bl = bx * bx + by * by + bz * bz;
    double adotb = ax * bx + ay * by + az * bz;
    double r11 = 1. / sqrt(al * bl);
    double costh = adotb * r11;
    double dudth, dthdcos;
    if (fabs(costh) >= 1.) {
      dthdcos = -1.;
      dudth = 0.;
    } else {
      double th = acos(costh);
      double dth = th - ep[b].x;
      dudth = ep[b].y * dth;
      dthdcos = -1. / sqrt(1. - costh * costh);
    }
    double dudcos = dudth * dthdcos;
    double d1x = costh * ax / al - bx * r11, d1y = costh * ay / al - by * r11, d1z = costh * az / al - bz * r11;
    double d3x = costh * bx / bl - ax * r11, d3y = costh * by / bl - ay * r11, d3z = costh * bz / bl - az * r11;
    fxa[i] += dudcos * d1x; fxa[n + i] += dudcos * d1y; fxa[2 * n + i] += dudcos * d1z;
    fxa[j] += dudcos * (-d1x - d3x); fxa[n + j] += dudcos * (-d1y - d3y); fxa[2 * n + j] += dudcos * (-d1z - d3z);
    fxa[k] += dudcos * d3x; fxa[n + k] += dudcos * d3y; fxa[2 * n + k] += dudcos * d3z;
  }
}

// force(2) alone: bonds + bends of every group into fxa, then rmass
__global__ void k_bonded(StepP P, const int *__restrict__ gaoff, const int *__restrict__ gatoms,
                         const double *__restrict__ pos, const double *__restrict__ mass, double *__restrict__ fxa,
                         const int *__restrict__ gboff, const int4 *__restrict__ bij, const double2 *__restrict__ bp,
                         const int *__restrict__ geoff, const int4 *__restrict__ eijk, const double2 *__restrict__ ep) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P.ngroups) return;
  const int n = P.n;
  for (int a = gaoff[g]; a < gaoff[g + 1]; a++) {
    int i = gatoms[a];
    fxa[i] = fxa[n + i] = fxa[2 * n + i] = 0.;
  }
  group_bonded(g, n, pos, fxa, gboff, bij, bp, geoff, eijk, ep);
  for (int a = gaoff[g]; a < gaoff[g + 1]; a++) {
    int i = gatoms[a];
    double r = 1. / mass[i];
    fxa[i] *= r; fxa[n + i] *= r; fxa[2 * n + i] *= r;
  }
}

// One pass of md_step.c:95-136 for level `intr`: the kick with the
// nonbonded accelerations, the ninrra x ninnra inner loop with force(2) on
// this group, then nrefsh's displacement test.
__global__ void k_inner(StepP P, int intr, const int *__restrict__ gaoff, const int *__restrict__ gatoms,
                        double *__restrict__ pos, double *__restrict__ vel, const double *__restrict__ mass,
                        const double *__restrict__ fxl, const double *__restrict__ fxs, double *__restrict__ fxa,
                        const double *__restrict__ dxn, const int *__restrict__ gboff,
                        const int4 *__restrict__ bij, const double2 *__restrict__ bp,
                        const int *__restrict__ geoff, const int4 *__restrict__ eijk,
                        const double2 *__restrict__ ep, const SysP *__restrict__ sp,
                        const int *__restrict__ sys_of, int *__restrict__ sreb, int *__restrict__ istate,
                        const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g == 0) istate[IS_INTR] = intr;
  if (g >= P.ngroups) return;
  const int n = P.n;
  const int a0 = gaoff[g], a1 = gaoff[g + 1];
  // long and short range intermolecular kick (md_step.c:97-103)
  for (int a = a0; a < a1; a++) {
    int i = gatoms[a];
    for (int d = 0; d < 3; d++) {
      int x = d * n + i;
      if (intr == 0) vel[x] += P.dter * fxl[x] + (P.use_fxs ? P.dter1 * fxs[x] : 0.0);
      else vel[x] += P.dts2 * fxs[x];
    }
  }
  const bool bonded = gboff[g + 1] > gboff[g] || geoff[g + 1] > geoff[g];
  for (int inrra = 0; inrra < P.ninrra; inrra++) {
    // the torsion level (fxr) is empty in this engine
    for (int intra = 0; intra < P.ninnra; intra++) {
      for (int a = a0; a < a1; a++) {
        int i = gatoms[a];
        for (int d = 0; d < 3; d++) {
          int x = d * n + i;
          vel[x] += P.dta2 * fxa[x];
          pos[x] += P.dta2 * vel[x];
          pos[x] += P.dta2 * vel[x];
        }
      }
      if (bonded) {
        for (int a = a0; a < a1; a++) {
          int i = gatoms[a];
          fxa[i] = fxa[n + i] = fxa[2 * n + i] = 0.;
        }
        group_bonded(g, n, pos, fxa, gboff, bij, bp, geoff, eijk, ep);
        for (int a = a0; a < a1; a++) {
          int i = gatoms[a];
          double r = 1. / mass[i];
          fxa[i] *= r; fxa[n + i] *= r; fxa[2 * n + i] *= r;
        }
      }
      for (int a = a0; a < a1; a++) {
        int i = gatoms[a];
        for (int d = 0; d < 3; d++) vel[d * n + i] += P.dta2 * fxa[d * n + i];
      }
    }
  }
  // nrefsh: any |r - r_last|^2 > skin^2/4 (md_finter.c:63-71), per system
  const int sy = sys_of[gatoms[a0]];
  const double skin2q = sp[sy].skin2q;
  bool far = false;
  for (int a = a0; a < a1; a++) {
    int i = gatoms[a];
    double xc = dxn[i] - pos[i], yc = dxn[n + i] - pos[n + i], zc = dxn[2 * n + i] - pos[2 * n + i];
    if (xc * xc + yc * yc + zc * zc > skin2q) far = true;
  }
  if (far) {
    sreb[sy] = 1;
    istate[IS_REBUILD] = 1;
  }
}

// standalone displacement test (cm3d_nb_nrefsh)
__global__ void k_disp(int n, const SysP *__restrict__ sp, const int *__restrict__ sys_of,
                       const double *__restrict__ pos, const double *__restrict__ dxn, int *__restrict__ sreb,
                       int *__restrict__ istate) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int sy = sys_of[i];
  double xc = dxn[i] - pos[i], yc = dxn[n + i] - pos[n + i], zc = dxn[2 * n + i] - pos[2 * n + i];
  if (xc * xc + yc * yc + zc * zc > sp[sy].skin2q) {
    sreb[sy] = 1;
    istate[IS_REBUILD] = 1;
  }
}

// RESETPOS (md_finter.c:79-95): if a rebuild is due fewer than 3 steps after
// the system's previous one, pull every atom that moved more than skin/2
// back toward its position at the last rebuild (by CM3D's factor skin2/d^2)
__global__ void k_resetpos(int n, const SysP *__restrict__ sp, const int *__restrict__ sys_of,
                           const int *__restrict__ sreb, const int *__restrict__ slast, double *__restrict__ pos,
                           const double *__restrict__ dxn, const int *__restrict__ istate,
                           long long *__restrict__ stat, long long *__restrict__ sstat) {
  if (istate[IS_REBUILD] == 0 || istate[IS_HALT] != 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int sy = sys_of[i];
  if (sreb[sy] == 0 || istate[IS_ISTEP] - slast[sy] >= 3) return;
  if (i == sp[sy].a0) {
    atomicAdd((unsigned long long *)(stat + ST_RESETS), 1ull);
    sstat[(size_t)sy * SS_COUNT + SS_RESETS] += 1;
  }
  const double skin2q = sp[sy].skin2q;
  double xc = pos[i] - dxn[i], yc = pos[n + i] - dxn[n + i], zc = pos[2 * n + i] - dxn[2 * n + i];
  double d2 = xc * xc + yc * yc + zc * zc;
  if (d2 > skin2q) {
    double scale = skin2q / d2;
    pos[i] = dxn[i] + scale * xc;
    pos[n + i] = dxn[n + i] + scale * yc;
    pos[2 * n + i] = dxn[2 * n + i] + scale * zc;
  }
}

// start of force(1) (md_fcntr.c:64-73): zero fxl (and fxs), add the
// excluded-pair correction of every group (ecorr, md_ewald.c:385-453), and
// collect the group's bonded energies and virials (getvbond / getvbend; the
// bend virial is the one md_fbend.c always compiles, its tensor formed from
// absolute positions as there)
__global__ void k_group_init(StepP P, int zero_fxs, const int *__restrict__ gaoff, const int *__restrict__ gatoms,
                             const double *__restrict__ pos, const double *__restrict__ q,
                             double *__restrict__ fxl, double *__restrict__ fxs, const int *__restrict__ gcoff,
                             const int2 *__restrict__ cij, const int *__restrict__ gboff,
                             const int4 *__restrict__ bij, const double2 *__restrict__ bp,
                             const int *__restrict__ geoff, const int4 *__restrict__ eijk,
                             const double2 *__restrict__ ep, double *__restrict__ acc,
                             const SysP *__restrict__ sp, const int *__restrict__ sys_of,
                             const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = P.n;
  // ecorr: pot, prs, t0 t1 t2 t4 t5 t8 | bond: v, w, t0..t8 | bend: v, w, t0..t8
  double v[30];
#pragma unroll
  for (int k = 0; k < 30; k++) v[k] = 0.;
  int sy = -1;
  if (g < P.ngroups) {
    sy = sys_of[gatoms[gaoff[g]]];
    const double kappa = sp[sy].kappa, kappa2 = sp[sy].kappa2;
    for (int a = gaoff[g]; a < gaoff[g + 1]; a++) {
      int i = gatoms[a];
      fxl[i] = fxl[n + i] = fxl[2 * n + i] = 0.;
      if (zero_fxs) fxs[i] = fxs[n + i] = fxs[2 * n + i] = 0.;
    }
    const double sqrt_pi = 1. / sqrt(M_PI);
    for (int c = gcoff[g]; c < gcoff[g + 1]; c++) {
      int ii = cij[c].x, jj = cij[c].y;
      double xd = pos[ii] - pos[jj], yd = pos[n + ii] - pos[n + jj], zd = pos[2 * n + ii] - pos[2 * n + jj];
      double dis2 = xd * xd + yd * yd + zd * zd, dis = sqrt(dis2);
      double qijr = q[ii] * q[jj] / dis;
      double erfr = erf(dis * kappa);
      v[0] += -qijr * erfr;
      double dv = -qijr * (-2. * kappa * exp(-kappa2 * dis2) * sqrt_pi + erfr / dis);
      v[1] += dis * dv;
      dv /= dis;
      v[2] += dv * xd * xd; v[3] += dv * xd * yd; v[4] += dv * xd * zd;
      v[5] += dv * yd * yd; v[6] += dv * yd * zd; v[7] += dv * zd * zd;
      xd *= dv; yd *= dv; zd *= dv;
      fxl[ii] += xd; fxl[n + ii] += yd; fxl[2 * n + ii] += zd;
      fxl[jj] -= xd; fxl[n + jj] -= yd; fxl[2 * n + jj] -= zd;
    }
    // getvbond (md_fbond.c:160-207), harmonic
    for (int b = gboff[g]; b < gboff[g + 1]; b++) {
      const int i = bij[b].x, j = bij[b].y;
      double dx = pos[i] - pos[j], dy = pos[n + i] - pos[n + j], dz = pos[2 * n + i] - pos[2 * n + j];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      double dr = r - bp[b].x;
      double fk = bp[b].y;
      v[8] += .5 * fk * dr * dr;
      fk = fk * dr / r;
      v[9] -= fk * r * r;
      v[10] -= fk * dx * dx; v[11] -= fk * dy * dx; v[12] -= fk * dz * dx;
      v[13] -= fk * dx * dy; v[14] -= fk * dy * dy; v[15] -= fk * dz * dy;
      v[16] -= fk * dx * dz; v[17] -= fk * dy * dz; v[18] -= fk * dz * dz;
    }
    // getvbend (md_fbend.c:295-330), harmonic; its virial needs -DPRESSURE
    for (int b = geoff[g]; b < geoff[g + 1]; b++) {
      const int i = eijk[b].x, j = eijk[b].y, k = eijk[b].z;
      double ax = pos[i] - pos[j], ay = pos[n + i] - pos[n + j], az = pos[2 * n + i] - pos[2 * n + j];
      double al = ax * ax + ay * ay + az * az;
      double bx = pos[k] - pos[j], by = pos[n + k] - pos[n + j], bz = pos[2 * n + k] - pos[2 * n + j];
      double bl = bx * bx + by * by + bz * bz;
      double r11 = 1. / sqrt(al * bl), costh = (ax * bx + ay * by + az * bz) * r11;
      costh = costh < 1. ? costh : 1.;
      costh = costh > -1. ? costh : -1.;
      double th = fabs(costh) >= 1. ? 1. : acos(costh);
      double dth = th - ep[b].x;
      v[19] += .5 * ep[b].y * dth * dth;
      // bend virial (md_fbend.c:322-398), harmonic: dU/dth = 0 at |cos| = 1
      const double dudth = fabs(costh) >= 1. ? 0. : ep[b].y * dth;
      const double dthdcos = fabs(costh) >= 1. ? -1. : -1. / sqrt(1. - costh * costh);
      const double dudcos = dudth * dthdcos;
      const double c1x = costh * ax / al - bx * r11, c1y = costh * ay / al - by * r11,
                   c1z = costh * az / al - bz * r11;
      const double c2x = -costh * (ax / al + bx / bl) + (ax + bx) * r11;
      const double c2y = -costh * (ay / al + by / bl) + (ay + by) * r11;
      const double c2z = -costh * (az / al + bz / bl) + (az + bz) * r11;
      const double c3x = costh * bx / bl - ax * r11, c3y = costh * by / bl - ay * r11,
                   c3z = costh * bz / bl - az * r11;
      const double xi = pos[i], xj = pos[j], xk = pos[k];
      const double yi = pos[n + i], yj = pos[n + j], yk = pos[n + k];
      const double zi = pos[2 * n + i], zj = pos[2 * n + j], zk = pos[2 * n + k];
      v[20] += dudcos * (ax * c1x + ay * c1y + az * c1z - bx * c3x - by * c3y - bz * c3z);
      v[21] += dudcos * (xi * c1x + xj * c2x + xk * c3x);
      v[22] += dudcos * (yi * c1x + yj * c2x + yk * c3x);
      v[23] += dudcos * (zi * c1x + zj * c2x + zk * c3x);
      v[24] += dudcos * (xi * c1y + xj * c2y + xk * c3y);
      v[25] += dudcos * (yi * c1y + yj * c2y + yk * c3y);
      v[26] += dudcos * (zi * c1y + zj * c2y + zk * c3y);
      v[27] += dudcos * (xi * c1z + xj * c2z + xk * c3z);
      v[28] += dudcos * (yi * c1z + yj * c2z + yk * c3z);
      v[29] += dudcos * (zi * c1z + zj * c2z + zk * c3z);
    }
  }
  const int slots[30] = {ACC_POT_ECORR, ACC_PRS_ECORR, ACC_PRS_ECORRT + 0, ACC_PRS_ECORRT + 1,
                         ACC_PRS_ECORRT + 2, ACC_PRS_ECORRT + 4, ACC_PRS_ECORRT + 5, ACC_PRS_ECORRT + 8,
                         ACC_VBOND, ACC_WBOND, ACC_WBONDT + 0, ACC_WBONDT + 1, ACC_WBONDT + 2,
                         ACC_WBONDT + 3, ACC_WBONDT + 4, ACC_WBONDT + 5, ACC_WBONDT + 6, ACC_WBONDT + 7,
                         ACC_WBONDT + 8, ACC_VBEND, ACC_WBEND, ACC_WBENDT + 0, ACC_WBENDT + 1,
                         ACC_WBENDT + 2, ACC_WBENDT + 3, ACC_WBENDT + 4, ACC_WBENDT + 5, ACC_WBENDT + 6,
                         ACC_WBENDT + 7, ACC_WBENDT + 8};
  sys_acc<30>(v, sy, acc, slots);
}

// end of force(1) / force(0): rmass (utils/md_util.new.c:219) and, inside
// step(), the closing kick of md_step.c:139-145; then the kinetic tensor of
// get_p2mt (md_fcntr.c:332-354) for geteng
__global__ void k_finish(int n, int level, int kick, int rm_l, int rm_s, double dk_l, double dk_s,
                         const double *__restrict__ mass, double *__restrict__ fxl, double *__restrict__ fxs,
                         double *__restrict__ vel, double *__restrict__ acc, int *__restrict__ istate,
                         int advance_step, const int *__restrict__ sys_of, int batch,
                         const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[6] = {0, 0, 0, 0, 0, 0};
  int sy = -1;
  if (i < n) {
    sy = sys_of[i];
    double r = 1. / mass[i];
    for (int d = 0; d < 3; d++) {
      int x = d * n + i;
      if (rm_l) fxl[x] *= r;
      if (rm_s) fxs[x] *= r;
      if (kick) {
        if (level == 1) vel[x] += dk_l * fxl[x] + (rm_s ? dk_s * fxs[x] : 0.0);
        else vel[x] += dk_s * fxs[x];
      }
    }
    double m = mass[i], vx = vel[i], vy = vel[n + i], vz = vel[2 * n + i];
    v[0] = m * (vx * vx);
    v[1] = m * (vy * vx);
    v[2] = m * (vz * vx);
    v[3] = m * (vy * vy);
    v[4] = m * (vz * vy);
    v[5] = m * (vz * vz);
  }
  if (i == 0 && advance_step) istate[IS_ISTEP] += 1;
  if (level == 1) {
    const int slots[6] = {ACC_P2MT + 0, ACC_P2MT + 1, ACC_P2MT + 2, ACC_P2MT + 4, ACC_P2MT + 5, ACC_P2MT + 8};
    if (batch) sys_acc<6>(v, sy, acc, slots);
    else block_acc<6>(v, acc, slots);
  }
}

// ------------------------------------------------------------------ host
static StepP step_params(Ctx *c) {
  StepP P;
  P.n = c->n;
  P.ngroups = c->ngroups;
  P.ninrra = c->nres_tors;
  P.ninnra = c->nres_intra;
  // md_step.c:73-78
  double dtl2 = .5 * c->dt;
  P.dts2 = dtl2 / (double)c->nres_lrf;
  P.dtr2 = P.dts2 / (double)c->nres_tors;
  P.dta2 = P.dtr2 / (double)c->nres_intra;
  P.dter = (double)c->nres_lrf * P.dts2;
  P.dter1 = (double)(1 - c->nres_lrf) * P.dts2;
  P.skin2q = .25 * c->skin * c->skin;
  P.kappa = c->kappa;
  P.kappa2 = c->kappa2;
  P.use_fxs = c->nres_lrf > 1 || c->need_short;
  return P;
}

struct UF {
  std::vector<int> p;
  explicit UF(int n) : p(n) { std::iota(p.begin(), p.end(), 0); }
  int f(int x) {
    while (p[x] != x) x = p[x] = p[p[x]];
    return x;
  }
  void u(int a, int b) {
    a = f(a);
    b = f(b);
    if (a != b) p[a < b ? b : a] = a < b ? a : b;
  }
};

int step_setup(Ctx *c, const cm3d_nb_system *systems, int nsys) {
  const int n = c->n;
  // every system's bonds, bends and excluded Ewald pairs with global atom
  // indices, in system order (CM3D's order inside a system)
  std::vector<int4> mb, me;            // {i, j, -, -} / {i, j, k, -}
  std::vector<double2> mbp, mep;       // {eq, fk}
  std::vector<int2> mc;
  for (int sy = 0; sy < nsys; sy++) {
    const cm3d_nb_system *s = systems + sy;
    const int a0 = c->h_sp[sy].a0;
    for (int b = 0; b < s->nbonds; b++) {
      int t = s->idxbond[b];
      if (s->itypbond[t] != 0) {
        set_error("system %d bond %d: only harmonic bonds are supported (itypbond %d)", sy, b, s->itypbond[t]);
        return CM3D_NB_ERR_ARG;
      }
      mb.push_back(make_int4(a0 + s->ibond[b], a0 + s->jbond[b], 0, 0));
      mbp.push_back(make_double2(s->eqbond[t], s->fkbond[t]));
    }
    for (int b = 0; b < s->nbends; b++) {
      int t = s->idxbend[b];
      if (s->itypbend[t] != 0) {
        set_error("system %d bend %d: only harmonic bends are supported (itypbend %d)", sy, b, s->itypbend[t]);
        return CM3D_NB_ERR_ARG;
      }
      me.push_back(make_int4(a0 + s->ibend[b], a0 + s->jbend[b], a0 + s->kbend[b], 0));
      mep.push_back(make_double2(s->eqbend[t], s->fkbend[t]));
    }
    for (int b = 0; b < s->necorr; b++) mc.push_back(make_int2(a0 + s->iecorr[b], a0 + s->jecorr[b]));
  }
  const int nb = (int)mb.size(), ne = (int)me.size(), nc = (int)mc.size();
  UF uf(n);
  for (int b = 0; b < nb; b++) uf.u(mb[b].x, mb[b].y);
  for (int b = 0; b < ne; b++) {
    uf.u(me[b].x, me[b].y);
    uf.u(me[b].y, me[b].z);
  }
  for (int b = 0; b < nc; b++) uf.u(mc[b].x, mc[b].y);
  // groups numbered by their lowest atom
  std::vector<int> gid(n, -1), root_gid(n, -1);
  int ng = 0;
  for (int i = 0; i < n; i++) {
    int r = uf.f(i);
    if (root_gid[r] < 0) root_gid[r] = ng++;
    gid[i] = root_gid[r];
  }
  c->ngroups = ng;
  std::vector<int> aoff(ng + 1, 0), atoms(n);
  for (int i = 0; i < n; i++) aoff[gid[i] + 1]++;
  for (int g = 0; g < ng; g++) aoff[g + 1] += aoff[g];
  {
    std::vector<int> cur(aoff.begin(), aoff.end() - 1);
    for (int i = 0; i < n; i++) atoms[cur[gid[i]]++] = i;
  }
  // bonds / bends / ecorr pairs grouped, CM3D's order kept inside a group
  std::vector<int> boff(ng + 1, 0), eoff(ng + 1, 0), coff(ng + 1, 0);
  for (int b = 0; b < nb; b++) boff[gid[mb[b].x] + 1]++;
  for (int b = 0; b < ne; b++) eoff[gid[me[b].y] + 1]++;
  for (int b = 0; b < nc; b++) coff[gid[mc[b].x] + 1]++;
  for (int g = 0; g < ng; g++) {
    boff[g + 1] += boff[g];
    eoff[g + 1] += eoff[g];
    coff[g + 1] += coff[g];
  }
  std::vector<int4> bij(nb > 0 ? nb : 1), eijk(ne > 0 ? ne : 1);
  std::vector<double2> bp(bij.size()), ep(eijk.size());
  std::vector<int2> cij(nc > 0 ? nc : 1), cpair(cij.size());
  {
    std::vector<int> cb(boff.begin(), boff.end() - 1), ce(eoff.begin(), eoff.end() - 1),
        cc(coff.begin(), coff.end() - 1);
    for (int b = 0; b < nb; b++) {
      int slot = cb[gid[mb[b].x]]++;
      bij[slot] = mb[b];
      bp[slot] = mbp[b];
    }
    for (int b = 0; b < ne; b++) {
      int slot = ce[gid[me[b].y]]++;
      eijk[slot] = me[b];
      ep[slot] = mep[b];
    }
    for (int b = 0; b < nc; b++) {
      int slot = cc[gid[mc[b].x]]++;
      cij[slot] = mc[b];
      cpair[b] = mc[b];
    }
  }
  CK(cudaMalloc(&c->grp_atom_off, sizeof(int) * (ng + 1)));
  CK(cudaMalloc(&c->grp_atoms, sizeof(int) * (size_t)n));
  CK(cudaMalloc(&c->grp_bond_off, sizeof(int) * (ng + 1)));
  CK(cudaMalloc(&c->grp_bend_off, sizeof(int) * (ng + 1)));
  CK(cudaMalloc(&c->grp_ecorr_off, sizeof(int) * (ng + 1)));
  CK(cudaMalloc(&c->bond_ij, sizeof(int4) * bij.size()));
  CK(cudaMalloc(&c->bond_p, sizeof(double2) * bp.size()));
  CK(cudaMalloc(&c->bend_ijk, sizeof(int4) * eijk.size()));
  CK(cudaMalloc(&c->bend_p, sizeof(double2) * ep.size()));
  CK(cudaMalloc(&c->ecorr_ij, sizeof(int2) * cij.size()));
  CK(cudaMalloc(&c->ecorr_pairs, sizeof(int2) * cpair.size()));
  CK(cudaMemcpy(c->grp_atom_off, aoff.data(), sizeof(int) * (ng + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->grp_atoms, atoms.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->grp_bond_off, boff.data(), sizeof(int) * (ng + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->grp_bend_off, eoff.data(), sizeof(int) * (ng + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->grp_ecorr_off, coff.data(), sizeof(int) * (ng + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->bond_ij, bij.data(), sizeof(int4) * bij.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->bond_p, bp.data(), sizeof(double2) * bp.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->bend_ijk, eijk.data(), sizeof(int4) * eijk.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->bend_p, ep.data(), sizeof(double2) * ep.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->ecorr_ij, cij.data(), sizeof(int2) * cij.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->ecorr_pairs, cpair.data(), sizeof(int2) * cpair.size(), cudaMemcpyHostToDevice));
  return CM3D_NB_OK;
}

int run_bonded(Ctx *c) {
  StepP P = step_params(c);
  const int B = 128;
  k_bonded<<<grid_for(c->ngroups, B), B, 0, c->st>>>(P, c->grp_atom_off, c->grp_atoms, c->pos, c->mass, c->fxa,
                                                     c->grp_bond_off, c->bond_ij, c->bond_p, c->grp_bend_off,
                                                     c->bend_ijk, c->bend_p);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

int group_init(Ctx *c, bool zero_fxs) {
  StepP P = step_params(c);
  const int B = 128;
  cudaEvent_t e0;
  tbegin(c, 3, &e0);
  k_group_init<<<grid_for(c->ngroups, B), B, 0, c->st>>>(P, zero_fxs ? 1 : 0, c->grp_atom_off, c->grp_atoms,
                                                         c->pos, c->q, c->fxl, c->fxs, c->grp_ecorr_off,
                                                         c->ecorr_ij, c->grp_bond_off, c->bond_ij, c->bond_p,
                                                         c->grp_bend_off, c->bend_ijk, c->bend_p, c->acc, c->sp,
                                                         c->sys_of, c->gate);
  tend(c, 3, e0);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

int finish_level1(Ctx *c, double dter, double dter1, bool kick) {
  const int B = 256;
  bool rs = c->need_short || c->nres_lrf > 1;
  k_finish<<<grid_for(c->n, B), B, 0, c->st>>>(c->n, 1, kick ? 1 : 0, 1, rs ? 1 : 0, dter, dter1, c->mass, c->fxl,
                                               c->fxs, c->vel, c->acc, c->istate, kick ? 1 : 0, c->sys_of,
                                               c->nsys > 1, c->gate);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

static int finish_level0(Ctx *c, double dts2, bool kick) {
  k_finish<<<grid_for(c->n, 256), 256, 0, c->st>>>(c->n, 0, kick ? 1 : 0, 0, 1, 0, dts2, c->mass, c->fxl, c->fxs,
                                                   c->vel, c->acc, c->istate, 0, c->sys_of, c->nsys > 1, c->gate);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

// clear the rebuild requests (the any-system flag and every system's own)
static int clear_rebuild(Ctx *c) {
  CK(cudaMemsetAsync(c->istate + IS_REBUILD, 0, sizeof(int), c->st));
  CK(cudaMemsetAsync(c->sreb, 0, sizeof(int) * (size_t)c->nsys, c->st));
  return CM3D_NB_OK;
}

int check_displacement(Ctx *c) {
  int rc;
  if ((rc = clear_rebuild(c))) return rc;
  k_disp<<<grid_for(c->n, 256), 256, 0, c->st>>>(c->n, c->sp, c->sys_of, c->pos, c->dxn, c->sreb, c->istate);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

int reset_positions(Ctx *c) {
  k_resetpos<<<grid_for(c->n, 256), 256, 0, c->st>>>(c->n, c->sp, c->sys_of, c->sreb, c->slast, c->pos, c->dxn,
                                                      c->istate, c->stat, c->sstat);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

// zero every accumulator force(1) and getvireal fill, in every system
static int zero_acc(Ctx *c) {
  CK(cudaMemset2DAsync(c->acc, sizeof(double) * ACC_STRIDE, 0, sizeof(double) * ACC_COUNT, (size_t)c->nsys, c->st));
  return CM3D_NB_OK;
}

// force(iflg) of md_fcntr.c:44-134 (levels 0, 1, 2)
int run_force(Ctx *c, int iflg) {
  int rc;
  if (iflg == 2) return run_bonded(c);
  if (!c->lists_built) {
    set_error("force(%d) before get_ngbr(): the pair lists do not exist yet", iflg);
    return CM3D_NB_ERR_STATE;
  }
  if (iflg == 1) {
    if ((rc = zero_acc(c))) return rc;
    if ((rc = group_init(c, true))) return rc;
    if ((rc = pair_forces(c, 1, 3))) return rc;
    if ((rc = kspace_forces(c))) return rc;
    return finish_level1(c, 0, 0, false);
  }
  if (iflg == 0) {
    CK(cudaMemsetAsync(c->fxs, 0, sizeof(double) * 3 * (size_t)c->n, c->st));
    if ((rc = pair_forces(c, 0, 3))) return rc;
    return finish_level0(c, 0, false);
  }
  set_error("force(): unknown level %d", iflg);
  return CM3D_NB_ERR_ARG;
}

// the nonbonded level that closes RESPA level `intr` (md_step.c:138-146):
// force(1) + kick on the last level, force(0) + kick otherwise
static int close_level(Ctx *c, int intr) {
  int rc;
  StepP P = step_params(c);
  if (intr == c->nres_lrf - 1) {
    if ((rc = zero_acc(c))) return rc;
    if ((rc = group_init(c, P.use_fxs))) return rc;
    if ((rc = pair_forces(c, 1, 3))) return rc;
    if ((rc = kspace_forces(c))) return rc;
    return finish_level1(c, P.dter, P.dter1, true);
  }
  CK(cudaMemsetAsync(c->fxs, 0, sizeof(double) * 3 * (size_t)c->n, c->st));
  if ((rc = pair_forces(c, 0, 3))) return rc;
  return finish_level0(c, P.dts2, true);
}

// RESPA level `intr` of one outer step (md_step.c:95-146); with `gated` the
// rebuild kernels are gated on the device flag (graph capture), otherwise
// the host reads the flag and rebuilds
static int one_level(Ctx *c, int intr, bool gated) {
  int rc;
  StepP P = step_params(c);
  const int B = 128;
  if ((rc = clear_rebuild(c))) return rc;
  cudaEvent_t e0;
  tbegin(c, 3, &e0);
  k_inner<<<grid_for(c->ngroups, B), B, 0, c->st>>>(P, intr, c->grp_atom_off, c->grp_atoms, c->pos, c->vel,
                                                    c->mass, c->fxl, c->fxs, c->fxa, c->dxn, c->grp_bond_off,
                                                    c->bond_ij, c->bond_p, c->grp_bend_off, c->bend_ijk,
                                                    c->bend_p, c->sp, c->sys_of, c->sreb, c->istate, c->gate);
  tend(c, 3, e0);
  c->launches++;
  CKL(c);
  if ((rc = reset_positions(c))) return rc;
  if (gated) {
    if ((rc = build_lists(c, true, false))) return rc;
  } else {
    CK(cudaMemcpyAsync(c->h_istate, c->istate, sizeof(int) * IS_COUNT, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (c->h_istate[IS_REBUILD]) {
      if ((rc = build_lists(c, false, false))) return rc;
    }
  }
  return close_level(c, intr);
}

static int one_step(Ctx *c, bool gated) {
  for (int intr = 0; intr < c->nres_lrf; intr++) {
    int rc = one_level(c, intr, gated);
    if (rc) return rc;
  }
  return CM3D_NB_OK;
}

static int set_istep(Ctx *c, int istep) {
  c->h_istate[IS_ISTEP] = istep;
  CK(cudaMemcpyAsync(c->istate + IS_ISTEP, c->h_istate + IS_ISTEP, sizeof(int), cudaMemcpyHostToDevice, c->st));
  return CM3D_NB_OK;
}

// Launch `nsteps` outer steps from istep0.  Graph mode: the captured step is
// replayed nsteps times on the context's stream, the device state is copied
// back asynchronously and an event marks the end; nothing waits (finish_steps
// completes the call).  Eager mode runs the steps to completion here.
int launch_steps(Ctx *c, int istep0, int nsteps) {
  int rc;
  if (!c->lists_built || !c->forces_valid) {
    set_error("step() before step_init(): forces and lists are not set up");
    return CM3D_NB_ERR_STATE;
  }
  if (c->pending) {
    set_error("step: the previous asynchronous steps have not been finished (cm3d_nb_step_wait)");
    return CM3D_NB_ERR_STATE;
  }
  if (nsteps <= 0) return CM3D_NB_OK;
  if ((rc = set_istep(c, istep0))) return rc;
  cudaEvent_t e4;
  if (!c->use_graph || c->timing.on) {
    tbegin(c, 4, &e4);
    for (int s = 0; s < nsteps; s++)
      if ((rc = one_step(c, false))) return rc;
    tend(c, 4, e4);
    return CM3D_NB_OK;
  }
  // graph replay: one captured step, every kernel gated on the device state
  // (rebuild flag; halt after a list overflow)
  if (!c->graph) {
    cudaGraph_t g;
    long long l0 = c->launches;
    CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    c->gate = c->istate;
    rc = one_step(c, true);
    c->gate = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->st, &g);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    CK(cudaGraphInstantiate(&c->graph, g, 0));
    cudaGraphDestroy(g);
    c->graph_launches = c->launches - l0;
    c->launches = l0;
  }
  tbegin(c, 4, &e4);
  for (int s = 0; s < nsteps; s++) {
    CK(cudaGraphLaunch(c->graph, c->st));
    c->launches += c->graph_launches;
  }
  tend(c, 4, e4);
  CK(cudaMemcpyAsync(c->h_istate, c->istate, sizeof(int) * IS_COUNT, cudaMemcpyDeviceToHost, c->st));
  if (!c->step_ev) CK(cudaEventCreateWithFlags(&c->step_ev, cudaEventDisableTiming));
  CK(cudaEventRecord(c->step_ev, c->st));
  c->pending = true;
  c->pend_istep0 = istep0;
  c->pend_nsteps = nsteps;
  return CM3D_NB_OK;
}

// Wait for launched steps (if any) and check the device state: a device-side
// rebuild that outgrew a list halted its step -- that step stopped right
// after its list build and every later kernel did nothing.  Grow the
// buffers, finish the step on the host-driven path and run the rest.
int finish_steps(Ctx *c) {
  int rc;
  if (!c->pending) return CM3D_NB_OK;
  CK(cudaEventSynchronize(c->step_ev));
  c->pending = false;
  if (!c->h_istate[IS_HALT]) return CM3D_NB_OK;
  const int istep0 = c->pend_istep0, nsteps = c->pend_nsteps;
  c->overflows_host++;
  const int failed = c->h_istate[IS_ISTEP], intr = c->h_istate[IS_INTR];
  CK(cudaMemsetAsync(c->istate + IS_HALT, 0, sizeof(int), c->st));
  if ((rc = build_lists(c, false, false))) return rc;
  if ((rc = close_level(c, intr))) return rc;
  for (int lv = intr + 1; lv < c->nres_lrf; lv++)
    if ((rc = one_level(c, lv, false))) return rc;
  if (c->graph) cudaGraphExecDestroy(c->graph);   // it holds the old buffer addresses
  c->graph = nullptr;
  int done = failed + 1 - istep0;
  if (done < nsteps) return run_step(c, failed + 1, nsteps - done);
  return CM3D_NB_OK;
}

// step() nsteps times: launch and finish
int run_step(Ctx *c, int istep0, int nsteps) {
  int rc;
  if ((rc = launch_steps(c, istep0, nsteps))) return rc;
  return finish_steps(c);
}

// non-blocking completion test of launched steps (finishes them when done)
int query_steps(Ctx *c, int *done) {
  *done = 1;
  if (!c->pending) return CM3D_NB_OK;
  cudaError_t e = cudaEventQuery(c->step_ev);
  if (e == cudaErrorNotReady) {
    *done = 0;
    return CM3D_NB_OK;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaEventQuery");
  return finish_steps(c);
}

}  // namespace cm3d
