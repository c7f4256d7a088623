// nb_step.cu -- the RESPA step on the device.
//
// Restates step() (integrate/md_step.c:62-159) for NVE with the level
// structure ninter (nres_lrf) / ninrra (nres_tors) / ninnra (nres_intra), the
// force levels of force() (energy/control/md_fcntr.c:44-134), nrefsh()
// (energy/control/md_finter.c:43-108, with its RESETPOS pull-back) and the
// harmonic fbond/fbend of the inner level (energy/intra/md_fbond.c:76-125,
// md_fbend.c:126-260).
//
// The intramolecular terms beyond them -- cross bonds in the inner level
// (fbondx, energy/intra/md_fbocross.c:40-97), torsions and 1-4 pairs in the
// torsion level (ftors md_ftors.c:117-293, fonfo md_fonefour.c:70-157) -- and
// the frozen atoms of freeze_atom (energy/control/md_fcntr.c:311-329) follow
// the same scheme.
//
// Bonds, bends, cross bonds, torsions, 1-4 pairs and excluded-pair
// corrections only couple atoms of one molecule, so the atoms are
// partitioned into groups (connected components of those terms) and one
// thread owns a group: the whole inner loop -- every
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
  int nchain;         // Nose-Hoover chain length (NVT), 0 for NVE
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

// cross bonds of group g into fxa: fk (|ri - rj| - eq1)(|rj - rk| - eq2)
__device__ __forceinline__ void group_bondx(int g, int n, const double *__restrict__ pos, double *__restrict__ fxa,
                                            const IntraDev &X) {
  for (int b = X.bx_off[g]; b < X.bx_off[g + 1]; b++) {
    const int4 t = X.bx_ijk[b];
    const double4 p = X.bx_par[b];
    const int i = t.x, j = t.y, k = t.z;
    const double ax = pos[i] - pos[j], ay = pos[n + i] - pos[n + j], az = pos[2 * n + i] - pos[2 * n + j];
    const double al = sqrt(ax * ax + ay * ay + az * az);
    const double bx = pos[j] - pos[k], by = pos[n + j] - pos[n + k], bz = pos[2 * n + j] - pos[2 * n + k];
    const double bl = sqrt(bx * bx + by * by + bz * bz);
    const double dr1 = al - p.x, dr2 = bl - p.y;
    const double fr1 = p.z * dr2 / al, fr2 = p.z * dr1 / bl;
    fxa[i] += -fr1 * ax; fxa[n + i] += -fr1 * ay; fxa[2 * n + i] += -fr1 * az;
    fxa[j] += fr1 * ax - fr2 * bx; fxa[n + j] += fr1 * ay - fr2 * by; fxa[2 * n + j] += fr1 * az - fr2 * bz;
    fxa[k] += fr2 * bx; fxa[n + k] += fr2 * by; fxa[2 * n + k] += fr2 * bz;
  }
}

// One torsion i-j-k-l.  With a = ri - rj, b = rj - rk, c = rk - rl and the
// plane normals d = a x b, e = b x c: cos(phi) = d.e / (|d| |e|).  For atom m,
// dcos/dr_m = (dF_m - cos dG_m) / G with F = d.e and G = |d| |e|; g[m] holds
// dU/dcos times that, the negative of the force.  u4 and dudcos (dU/dcos / G)
// are kept for the virial's j-l term.
struct TorsTerm {
  double a[3], b[3], c[3], g[4][3], u4[3], dudcos, pot;
};

__device__ __forceinline__ void torsion_term(int n, const double *__restrict__ pos, int4 at, int2 par,
                                             const IntraDev &X, TorsTerm &T) {
  const int i = at.x, j = at.y, k = at.z, l = at.w;
  const double ax = pos[i] - pos[j], ay = pos[n + i] - pos[n + j], az = pos[2 * n + i] - pos[2 * n + j];
  const double bx = pos[j] - pos[k], by = pos[n + j] - pos[n + k], bz = pos[2 * n + j] - pos[2 * n + k];
  const double cx = pos[k] - pos[l], cy = pos[n + k] - pos[n + l], cz = pos[2 * n + k] - pos[2 * n + l];
  const double dx = ay * bz - az * by, dy = az * bx - ax * bz, dz = ax * by - ay * bx;
  const double dl = sqrt(dx * dx + dy * dy + dz * dz);
  const double ex = by * cz - bz * cy, ey = bz * cx - bx * cz, ez = bx * cy - by * cx;
  const double el = sqrt(ex * ex + ey * ey + ez * ez);
  const double cphi = (dx * ex + dy * ey + dz * ez) / (dl * el);
  double dudcos;
  if (par.x == 0) {
    // harmonic in phi; dU/dphi dphi/dcos, zero at |cos| = 1
    const double2 h = X.tor_h[par.y];
    double phi = 0., dphi;
    if (cphi >= 1.0 || cphi <= -1.0) {
      dphi = phi - h.x;
      dudcos = 0.;
    } else {
      phi = acos(cphi);
      dphi = phi - h.x;
      dudcos = (h.y * dphi) * (-1. / sqrt(1. - cphi * cphi));
    }
    T.pot = .5 * h.y * dphi * dphi;
  } else {
    // power series sum_m v_m cos^m (Horner's scheme for U and dU/dcos)
    const double *v = X.tor_v + (size_t)par.y * CM3D_NB_MAXPOWER_TORS;
    double tpot = v[CM3D_NB_MAXPOWER_TORS - 1];
    dudcos = ((double)CM3D_NB_MAXPOWER_TORS - 1.) * v[CM3D_NB_MAXPOWER_TORS - 1];
    for (int m = CM3D_NB_MAXPOWER_TORS - 2; m > 0; m--) dudcos = dudcos * cphi + v[m] * (double)m;
    for (int m = CM3D_NB_MAXPOWER_TORS - 2; m >= 0; m--) tpot = tpot * cphi + v[m];
    T.pot = tpot;
  }
  const double G = dl * el, dre = dl / el, erd = el / dl;
  dudcos *= 1. / G;
  T.dudcos = dudcos;
  T.a[0] = ax; T.a[1] = ay; T.a[2] = az;
  T.b[0] = bx; T.b[1] = by; T.b[2] = bz;
  T.c[0] = cx; T.c[1] = cy; T.c[2] = cz;
  // dF_m and dG_m of the four atoms (F and G differentiated by hand)
  const double f1x = by * ez - bz * ey, f1y = bz * ex - bx * ez, f1z = bx * ey - by * ex;
  const double f2x = (cy * dz - cz * dy + (az + bz) * ey - (ay + by) * ez);
  const double f2y = (cz * dx - cx * dz + (ax + bx) * ez - (az + bz) * ex);
  const double f2z = (cx * dy - cy * dx + (ay + by) * ex - (ax + bx) * ey);
  const double f3x = (ay * ez - az * ey + (bz + cz) * dy - (by + cy) * dz);
  const double f3y = (az * ex - ax * ez + (bx + cx) * dz - (bz + cz) * dx);
  const double f3z = (ax * ey - ay * ex + (by + cy) * dx - (bx + cx) * dy);
  const double f4x = by * dz - bz * dy, f4y = bz * dx - bx * dz, f4z = bx * dy - by * dx;
  const double h1x = (by * dz - bz * dy) * erd, h1y = (bz * dx - bx * dz) * erd, h1z = (bx * dy - by * dx) * erd;
  const double h2x = ((dy * (az + bz) - dz * (ay + by)) * erd + (cy * ez - cz * ey) * dre);
  const double h2y = ((dz * (ax + bx) - dx * (az + bz)) * erd + (cz * ex - cx * ez) * dre);
  const double h2z = ((dx * (ay + by) - dy * (ax + bx)) * erd + (cx * ey - cy * ex) * dre);
  const double h3x = ((ay * dz - az * dy) * erd + (ey * (bz + cz) - ez * (by + cy)) * dre);
  const double h3y = ((az * dx - ax * dz) * erd + (ez * (bx + cx) - ex * (bz + cz)) * dre);
  const double h3z = ((ax * dy - ay * dx) * erd + (ex * (by + cy) - ey * (bx + cx)) * dre);
  const double h4x = (by * ez - bz * ey) * dre, h4y = (bz * ex - bx * ez) * dre, h4z = (bx * ey - by * ex) * dre;
  T.g[0][0] = dudcos * (f1x - cphi * h1x); T.g[0][1] = dudcos * (f1y - cphi * h1y); T.g[0][2] = dudcos * (f1z - cphi * h1z);
  T.g[1][0] = dudcos * (f2x - cphi * h2x); T.g[1][1] = dudcos * (f2y - cphi * h2y); T.g[1][2] = dudcos * (f2z - cphi * h2z);
  T.g[2][0] = dudcos * (f3x - cphi * h3x); T.g[2][1] = dudcos * (f3y - cphi * h3y); T.g[2][2] = dudcos * (f3z - cphi * h3z);
  T.u4[0] = f4x - cphi * h4x; T.u4[1] = f4y - cphi * h4y; T.u4[2] = f4z - cphi * h4z;
  T.g[3][0] = dudcos * T.u4[0]; T.g[3][1] = dudcos * T.u4[1]; T.g[3][2] = dudcos * T.u4[2];
}

// quadratic interpolation of a 1-4 table at squared distance dis2; below the
// table's start the first knot is used and *under set (md_fonefour.c:125-128)
__device__ __forceinline__ double o14_interp(const double *__restrict__ tab, int2 tb, double4 rng, double dis2,
                                             bool *under) {
  double p = (dis2 - rng.x) * rng.z;
  int k = (int)p;
  if (k < 1) {
    *under = true;
    k = 1;
    p = 1.;
  }
  // CM3D's tables end three knots past rmax14 (dx2tab = (ntab - 3)/(rmax^2 -
  // rmin^2)), so k + 1 < ntab for every dis2 < rmax14^2; the clamp only
  // keeps other input in bounds
  k = k < tb.y - 2 ? k : tb.y - 2;
  p = p - (double)k;
  const double *v = tab + tb.x;
  const double fm1 = v[k - 1], f0 = v[k], f1 = v[k + 1];
  return f0 + .5 * p * (f1 - fm1 + p * (fm1 - 2. * f0 + f1));
}

// the torsion level of group g into fxr (raw forces): its torsions, then its
// 1-4 pairs (tabulated force times scale_onefour, bare Coulomb times
// scale_onefour_e, within rmax14)
__device__ __forceinline__ void group_tors_level(int g, int n, const double *__restrict__ pos,
                                                 const double *__restrict__ q, double *__restrict__ fxr,
                                                 const IntraDev &X, long long *__restrict__ stat) {
  if (!X.tor_off) return;
  for (int t = X.tor_off[g]; t < X.tor_off[g + 1]; t++) {
    const int4 at = X.tor_ijkl[t];
    TorsTerm T;
    torsion_term(n, pos, at, X.tor_par[t], X, T);
    const int ids[4] = {at.x, at.y, at.z, at.w};
#pragma unroll
    for (int m = 0; m < 4; m++) {
      fxr[ids[m]] -= T.g[m][0];
      fxr[n + ids[m]] -= T.g[m][1];
      fxr[2 * n + ids[m]] -= T.g[m][2];
    }
  }
  bool under = false;
  for (int o = X.o14_off[g]; o < X.o14_off[g + 1]; o++) {
    const int4 pr = X.o14_ij[o];
    const int i = pr.x, j = pr.y;
    double xd = pos[i] - pos[j], yd = pos[n + i] - pos[n + j], zd = pos[2 * n + i] - pos[2 * n + j];
    const double dis2 = xd * xd + yd * yd + zd * zd;
    const double4 rng = X.o14_rng[pr.z];
    if (!(dis2 < rng.y)) continue;
    double fcc = o14_interp(X.o14_dv, X.o14_tab[pr.z], rng, dis2, &under) * rng.w;
    const double qij = q[i] * q[j];
    if (qij != 0) fcc -= qij * X.o14_se[pr.z] / (sqrt(dis2) * dis2);
    xd *= fcc; yd *= fcc; zd *= fcc;
    fxr[i] -= xd; fxr[n + i] -= yd; fxr[2 * n + i] -= zd;
    fxr[j] += xd; fxr[n + j] += yd; fxr[2 * n + j] += zd;
  }
  if (under) atomicAdd((unsigned long long *)(stat + ST_UNDERFLOW), 1ull);
}

// freeze_atom for one atom after a force level: no velocity, and the level's
// force block zeroed (the other blocks already are: every level zeroes them)
__device__ __forceinline__ void freeze_one(int i, int n, double *__restrict__ vel, double *__restrict__ f) {
  vel[i] = vel[n + i] = vel[2 * n + i] = 0.;
  f[i] = f[n + i] = f[2 * n + i] = 0.;
}

// force(3) alone: torsions + 1-4 pairs of every group into fxr, rmass, freeze
__global__ void k_tors_level(StepP P, const int *__restrict__ gaoff, const int *__restrict__ gatoms,
                             const double *__restrict__ pos, const double *__restrict__ q,
                             const double *__restrict__ mass, double *__restrict__ vel, double *__restrict__ fxr,
                             IntraDev X, long long *__restrict__ stat) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P.ngroups) return;
  const int n = P.n;
  for (int a = gaoff[g]; a < gaoff[g + 1]; a++) {
    int i = gatoms[a];
    fxr[i] = fxr[n + i] = fxr[2 * n + i] = 0.;
  }
  group_tors_level(g, n, pos, q, fxr, X, stat);
  for (int a = gaoff[g]; a < gaoff[g + 1]; a++) {
    int i = gatoms[a];
    double r = 1. / mass[i];
    fxr[i] *= r; fxr[n + i] *= r; fxr[2 * n + i] *= r;
    if (X.frz && X.frz[i]) freeze_one(i, n, vel, fxr);
  }
}

// force(2) alone: bonds + bends + cross bonds of every group into fxa, then
// rmass and freeze
__global__ void k_bonded(StepP P, const int *__restrict__ gaoff, const int *__restrict__ gatoms,
                         const double *__restrict__ pos, const double *__restrict__ mass, double *__restrict__ vel,
                         double *__restrict__ fxa, const int *__restrict__ gboff, const int4 *__restrict__ bij,
                         const double2 *__restrict__ bp, const int *__restrict__ geoff,
                         const int4 *__restrict__ eijk, const double2 *__restrict__ ep, IntraDev X) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P.ngroups) return;
  const int n = P.n;
  for (int a = gaoff[g]; a < gaoff[g + 1]; a++) {
    int i = gatoms[a];
    fxa[i] = fxa[n + i] = fxa[2 * n + i] = 0.;
  }
  group_bonded(g, n, pos, fxa, gboff, bij, bp, geoff, eijk, ep);
  if (X.bx_off) group_bondx(g, n, pos, fxa, X);
  for (int a = gaoff[g]; a < gaoff[g + 1]; a++) {
    int i = gatoms[a];
    double r = 1. / mass[i];
    fxa[i] *= r; fxa[n + i] *= r; fxa[2 * n + i] *= r;
    if (X.frz && X.frz[i]) freeze_one(i, n, vel, fxa);
  }
}

// One pass of md_step.c:95-136 for level `intr`: the kick with the
// nonbonded accelerations, the ninrra x ninnra inner loop with force(2) on
// this group, then nrefsh's displacement test.
template <bool INTRA>
__global__ void k_inner(StepP P, int intr, const int *__restrict__ gaoff, const int *__restrict__ gatoms,
                        double *__restrict__ pos, double *__restrict__ vel, const double *__restrict__ mass,
                        const double *__restrict__ fxl, const double *__restrict__ fxs, double *__restrict__ fxa,
                        const double *__restrict__ dxn, const int *__restrict__ gboff,
                        const int4 *__restrict__ bij, const double2 *__restrict__ bp,
                        const int *__restrict__ geoff, const int4 *__restrict__ eijk,
                        const double2 *__restrict__ ep, const SysP *__restrict__ sp,
                        const int *__restrict__ sys_of, int *__restrict__ sreb, int *__restrict__ istate,
                        const int *__restrict__ gs, IntraDev X, const double *__restrict__ q,
                        double *__restrict__ fxr, long long *__restrict__ stat) {
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
  const bool has_bx = INTRA && X.bx_off && X.bx_off[g + 1] > X.bx_off[g];
  const bool bonded = gboff[g + 1] > gboff[g] || geoff[g + 1] > geoff[g] || has_bx;
  // a group without torsions or 1-4 pairs has fxr = 0: its torsion-level
  // kicks change nothing and are skipped
  const bool tors = INTRA && X.tor_off && (X.tor_off[g + 1] > X.tor_off[g] || X.o14_off[g + 1] > X.o14_off[g]);
  for (int inrra = 0; inrra < P.ninrra; inrra++) {
    if (tors) {
      for (int a = a0; a < a1; a++) {
        int i = gatoms[a];
        for (int d = 0; d < 3; d++) vel[d * n + i] += P.dtr2 * fxr[d * n + i];
      }
    }
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
        if (has_bx) group_bondx(g, n, pos, fxa, X);
        for (int a = a0; a < a1; a++) {
          int i = gatoms[a];
          double r = 1. / mass[i];
          fxa[i] *= r; fxa[n + i] *= r; fxa[2 * n + i] *= r;
          if (INTRA && X.frz && X.frz[i]) freeze_one(i, n, vel, fxa);
        }
      }
      for (int a = a0; a < a1; a++) {
        int i = gatoms[a];
        for (int d = 0; d < 3; d++) vel[d * n + i] += P.dta2 * fxa[d * n + i];
      }
    }
    // force(3) on this group, then the closing torsion-level kick
    if (tors) {
      for (int a = a0; a < a1; a++) {
        int i = gatoms[a];
        fxr[i] = fxr[n + i] = fxr[2 * n + i] = 0.;
      }
      group_tors_level(g, n, pos, q, fxr, X, stat);
      for (int a = a0; a < a1; a++) {
        int i = gatoms[a];
        double r = 1. / mass[i];
        fxr[i] *= r; fxr[n + i] *= r; fxr[2 * n + i] *= r;
        if (X.frz && X.frz[i]) freeze_one(i, n, vel, fxr);
        for (int d = 0; d < 3; d++) vel[d * n + i] += P.dtr2 * fxr[d * n + i];
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

// ---- NVT: the inner level with Nose-Hoover chains (intnhc_new,
// integrate/md_therm.new.c:278-333, called between the two half drifts of
// every inner substep, md_step.c:117).  The chain update needs every
// thermostat's kinetic sum, a reduction over all groups, so each inner
// substep runs as four launches: k_nvt_a (kicks, first half drift, the
// first velocity scaling, each atom's kinetic term), k_nvt_ksum (the
// thermostats' kinetic sums in a fixed order), k_nvt_chain (one thread per
// thermostat) and k_nvt_c (second scaling, second half drift, bonded
// forces, kicks and, at the level's end, the displacement test).

__device__ __forceinline__ double nhc_factor(int thm, int nchain, double dta2, const double *__restrict__ veta) {
  return exp(-dta2 * (thm >= 0 ? veta[(size_t)thm * nchain] : 0.));
}

__global__ void k_nvt_a(StepP P, int intr, int level_start, int tors_start, const int *__restrict__ gaoff,
                        const int *__restrict__ gatoms, double *__restrict__ pos, double *__restrict__ vel,
                        const double *__restrict__ mass, const double *__restrict__ fxl,
                        const double *__restrict__ fxs, const double *__restrict__ fxa,
                        const double *__restrict__ fxr, const int *__restrict__ ithm,
                        const double *__restrict__ veta, double *__restrict__ kin, IntraDev X,
                        int *__restrict__ istate, const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g == 0 && level_start) istate[IS_INTR] = intr;
  if (g >= P.ngroups) return;
  const int n = P.n;
  const bool tors = X.tor_off && (X.tor_off[g + 1] > X.tor_off[g] || X.o14_off[g + 1] > X.o14_off[g]);
  for (int a = gaoff[g]; a < gaoff[g + 1]; a++) {
    const int i = gatoms[a];
    for (int d = 0; d < 3; d++) {
      const int x = d * n + i;
      if (level_start) {
        if (intr == 0) vel[x] += P.dter * fxl[x] + (P.use_fxs ? P.dter1 * fxs[x] : 0.0);
        else vel[x] += P.dts2 * fxs[x];
      }
      if (tors_start && tors) vel[x] += P.dtr2 * fxr[x];
      vel[x] += P.dta2 * fxa[x];
      pos[x] += P.dta2 * vel[x];
    }
    const int thm = ithm[i];
    const double e = nhc_factor(thm, P.nchain, P.dta2, veta);
    vel[i] *= e;
    vel[n + i] *= e;
    vel[2 * n + i] *= e;
    // this atom's kinetic term; k_nvt_ksum adds them per thermostat in a
    // fixed order (atoms without a thermostat are in no chunk)
    kin[i] = mass[i] * (vel[i] * vel[i] + vel[n + i] * vel[n + i] + vel[2 * n + i] * vel[2 * n + i]);
  }
}

// the kinetic sums of the thermostats' chunks: one warp per chunk, a lane-
// strided sum and the warp's fixed shuffle tree (the same order every step,
// alone or in a batch)
__global__ void k_nvt_ksum(int nchunks, const int2 *__restrict__ chunk, const int *__restrict__ atoms,
                           const double *__restrict__ kin, double *__restrict__ chsum, const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  const int ch = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (ch >= nchunks) return;
  const int2 r = chunk[ch];
  double s = 0.0;
  for (int k = r.x + lane; k < r.y; k += 32) s += kin[atoms[k]];
  s = warp_sum(s);
  if (lane == 0) chsum[ch] = s;
}

// the chain half step of one thermostat, in intnhc_new's order: links from
// the top, forces (forcen_new, md_therm.new.c:175-198), velocities and
// positions, the recurrence, links from the bottom
__global__ void k_nvt_chain(int ntherm, int nchain, double dta2, double *__restrict__ nhc,
                            const double *__restrict__ chsum, const int *__restrict__ choff,
                            const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ntherm) return;
  const size_t tc = (size_t)ntherm * nchain, o = (size_t)j * nchain;
  const double *m = nhc + o, *gk = nhc + tc + o;
  double *eta = nhc + 2 * tc + o, *v = nhc + 3 * tc + o, *f = nhc + 4 * tc + o;
  const double dta = 2. * dta2;
  for (int i = 0; i < nchain - 1; i++) v[i] *= exp(-dta2 * v[i + 1]);
  double p2m = 0.0;
  for (int k = choff[j]; k < choff[j + 1]; k++) p2m += chsum[k];
  f[0] = (p2m - gk[0]) / m[0];
  for (int i = 1; i < nchain; i++) f[i] = (m[i - 1] * v[i - 1] * v[i - 1] - gk[i]) / m[i];
  for (int i = 0; i < nchain; i++) v[i] += dta2 * f[i];
  for (int i = 0; i < nchain; i++) eta[i] += dta * v[i];
  v[0] += dta2 * f[0];
  for (int i = 1; i < nchain; i++) v[i] += dta2 * (m[i - 1] * v[i - 1] * v[i - 1] - gk[i]) / m[i];
  for (int i = nchain - 2; i >= 0; i--) v[i] *= exp(-dta2 * v[i + 1]);
}

__global__ void k_nvt_c(StepP P, int tors_end, int level_end, const int *__restrict__ gaoff,
                        const int *__restrict__ gatoms, double *__restrict__ pos, double *__restrict__ vel,
                        const double *__restrict__ mass, const double *__restrict__ q, double *__restrict__ fxa,
                        double *__restrict__ fxr, const double *__restrict__ dxn, const int *__restrict__ gboff,
                        const int4 *__restrict__ bij, const double2 *__restrict__ bp,
                        const int *__restrict__ geoff, const int4 *__restrict__ eijk,
                        const double2 *__restrict__ ep, const int *__restrict__ ithm,
                        const double *__restrict__ veta, const SysP *__restrict__ sp,
                        const int *__restrict__ sys_of, int *__restrict__ sreb, int *__restrict__ istate,
                        IntraDev X, long long *__restrict__ stat, const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P.ngroups) return;
  const int n = P.n;
  const int a0 = gaoff[g], a1 = gaoff[g + 1];
  const bool has_bx = X.bx_off && X.bx_off[g + 1] > X.bx_off[g];
  const bool bonded = gboff[g + 1] > gboff[g] || geoff[g + 1] > geoff[g] || has_bx;
  const bool tors = X.tor_off && (X.tor_off[g + 1] > X.tor_off[g] || X.o14_off[g + 1] > X.o14_off[g]);
  for (int a = a0; a < a1; a++) {
    const int i = gatoms[a];
    const double e = nhc_factor(ithm[i], P.nchain, P.dta2, veta);
    for (int d = 0; d < 3; d++) {
      const int x = d * n + i;
      vel[x] *= e;
      pos[x] += P.dta2 * vel[x];
    }
  }
  if (bonded) {
    for (int a = a0; a < a1; a++) {
      const int i = gatoms[a];
      fxa[i] = fxa[n + i] = fxa[2 * n + i] = 0.;
    }
    group_bonded(g, n, pos, fxa, gboff, bij, bp, geoff, eijk, ep);
    if (has_bx) group_bondx(g, n, pos, fxa, X);
    for (int a = a0; a < a1; a++) {
      const int i = gatoms[a];
      const double r = 1. / mass[i];
      fxa[i] *= r; fxa[n + i] *= r; fxa[2 * n + i] *= r;
      if (X.frz && X.frz[i]) freeze_one(i, n, vel, fxa);
    }
  }
  for (int a = a0; a < a1; a++) {
    const int i = gatoms[a];
    for (int d = 0; d < 3; d++) vel[d * n + i] += P.dta2 * fxa[d * n + i];
  }
  if (tors_end && tors) {
    for (int a = a0; a < a1; a++) {
      const int i = gatoms[a];
      fxr[i] = fxr[n + i] = fxr[2 * n + i] = 0.;
    }
    group_tors_level(g, n, pos, q, fxr, X, stat);
    for (int a = a0; a < a1; a++) {
      const int i = gatoms[a];
      const double r = 1. / mass[i];
      fxr[i] *= r; fxr[n + i] *= r; fxr[2 * n + i] *= r;
      if (X.frz && X.frz[i]) freeze_one(i, n, vel, fxr);
      for (int d = 0; d < 3; d++) vel[d * n + i] += P.dtr2 * fxr[d * n + i];
    }
  }
  if (level_end) {
    const int sy = sys_of[gatoms[a0]];
    const double skin2q = sp[sy].skin2q;
    bool far = false;
    for (int a = a0; a < a1; a++) {
      const int i = gatoms[a];
      const double xc = dxn[i] - pos[i], yc = dxn[n + i] - pos[n + i], zc = dxn[2 * n + i] - pos[2 * n + i];
      if (xc * xc + yc * yc + zc * zc > skin2q) far = true;
    }
    if (far) {
      sreb[sy] = 1;
      istate[IS_REBUILD] = 1;
    }
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
// The molecules (groups) with intramolecular Coulomb corrections, bonds or
// bends, listed in gwork: their energies, virials and ecorr forces.  The
// force arrays are zeroed beforehand (group_init), so groups without such
// terms -- every atom of a monatomic fluid -- need no thread.
__global__ void k_group_init(StepP P, const int *__restrict__ gwork, int ngw, const int *__restrict__ gaoff,
                             const int *__restrict__ gatoms,
                             const double *__restrict__ pos, const double *__restrict__ q,
                             double *__restrict__ fxl, double *__restrict__ fxs, const int *__restrict__ gcoff,
                             const int2 *__restrict__ cij, const int *__restrict__ gboff,
                             const int4 *__restrict__ bij, const double2 *__restrict__ bp,
                             const int *__restrict__ geoff, const int4 *__restrict__ eijk,
                             const double2 *__restrict__ ep, double *__restrict__ acc,
                             const SysP *__restrict__ sp, const int *__restrict__ sys_of,
                             const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = P.n;
  // ecorr: pot, prs, t0 t1 t2 t4 t5 t8 | bond: v, w, t0..t8 | bend: v, w, t0..t8
  double v[30];
#pragma unroll
  for (int k = 0; k < 30; k++) v[k] = 0.;
  int sy = -1;
  if (gi < ngw) {
    const int g = gwork[gi];
    sy = sys_of[gatoms[gaoff[g]]];
    const double kappa = sp[sy].kappa, kappa2 = sp[sy].kappa2;
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

// energies and virials of the cross bonds, torsions and 1-4 pairs, per group
// (getvbondx md_fbocross.c:100-168, getvtors md_ftors.c:296-542 with its
// PRESSURE tensor, getvonfo md_fonefour.c:160-314).  The 1-4 sums are kept
// unscaled; the host applies scale_onefour / scale_onefour_e per system.
__global__ void k_intra_energy(StepP P, const int *__restrict__ gaoff, const int *__restrict__ gatoms,
                               const double *__restrict__ pos, const double *__restrict__ q, IntraDev X,
                               double *__restrict__ acc, const int *__restrict__ sys_of,
                               const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = P.n;
  // bondx: v, w, t[9] | tors: v, t[9] | onfo: v, w, t[9], v_e, t_e[9]
  double v[42];
#pragma unroll
  for (int k = 0; k < 42; k++) v[k] = 0.;
  int sy = -1;
  if (g < P.ngroups) {
    sy = sys_of[gatoms[gaoff[g]]];
    for (int b = X.bx_off[g]; b < X.bx_off[g + 1]; b++) {
      const int4 t = X.bx_ijk[b];
      const double4 p = X.bx_par[b];
      const double a3[3] = {pos[t.x] - pos[t.y], pos[n + t.x] - pos[n + t.y], pos[2 * n + t.x] - pos[2 * n + t.y]};
      const double b3[3] = {pos[t.y] - pos[t.z], pos[n + t.y] - pos[n + t.z], pos[2 * n + t.y] - pos[2 * n + t.z]};
      const double al = sqrt(a3[0] * a3[0] + a3[1] * a3[1] + a3[2] * a3[2]);
      const double bl = sqrt(b3[0] * b3[0] + b3[1] * b3[1] + b3[2] * b3[2]);
      const double dr1 = al - p.x, dr2 = bl - p.y, fk = p.z;
      v[0] += fk * dr1 * dr2;
      v[1] -= fk * (bl * dr1 + al * dr2);
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) v[2 + 3 * r + c] -= fk * (dr1 * b3[c] * b3[r] / bl + dr2 * a3[c] * a3[r] / al);
    }
    for (int t = X.tor_off[g]; t < X.tor_off[g + 1]; t++) {
      TorsTerm T;
      torsion_term(n, pos, X.tor_ijkl[t], X.tor_par[t], X, T);
      v[11] += T.pot;
      // the i-j, j-k and j-l separations times the forces on i, k and l
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          double w = v[12 + 3 * r + c];
          w -= T.a[r] * T.g[0][c];
          w += T.b[r] * T.g[2][c];
          w += (T.b[r] + T.c[r]) * T.dudcos * T.u4[c];
          v[12 + 3 * r + c] = w;
        }
    }
    bool under = false;
    for (int o = X.o14_off[g]; o < X.o14_off[g + 1]; o++) {
      const int4 pr = X.o14_ij[o];
      const int i = pr.x, j = pr.y;
      const double d[3] = {pos[i] - pos[j], pos[n + i] - pos[n + j], pos[2 * n + i] - pos[2 * n + j]};
      const double dis2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      const double4 rng = X.o14_rng[pr.z];
      if (!(dis2 < rng.y)) continue;
      const int2 tb = X.o14_tab[pr.z];
      v[21] += o14_interp(X.o14_v, tb, rng, dis2, &under);
      const double f = o14_interp(X.o14_dv, tb, rng, dis2, &under);
      v[22] -= dis2 * f;
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) v[23 + 3 * r + c] -= d[c] * d[r] * f;
      const double qij = q[i] * q[j];
      if (qij != 0) {
        const double fe = qij / sqrt(dis2);
        v[32] += fe;
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int c = 0; c < 3; c++) v[33 + 3 * r + c] += fe * d[c] * d[r] / dis2;
      }
    }
  }
  int slots[42];
  slots[0] = ACC_VBOND;
  slots[1] = ACC_WBOND;
  slots[11] = ACC_VTORS;
  slots[21] = ACC_VONFO;
  slots[22] = ACC_WONFO;
  slots[32] = ACC_VONFO_E;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    slots[2 + k] = ACC_WBONDXT + k;
    slots[12 + k] = ACC_WTORST + k;
    slots[23 + k] = ACC_WONFOT + k;
    slots[33 + k] = ACC_WONFOET + k;
  }
  sys_acc<42>(v, sy, acc, slots);
}

// end of force(1) / force(0): rmass (utils/md_util.new.c:219) and, inside
// step(), the closing kick of md_step.c:139-145; then the kinetic tensor of
// get_p2mt (md_fcntr.c:332-354) for geteng
__global__ void k_finish(int n, int level, int kick, int rm_l, int rm_s, double dk_l, double dk_s,
                         const double *__restrict__ mass, double *__restrict__ fxl, double *__restrict__ fxs,
                         double *__restrict__ vel, double *__restrict__ acc, int *__restrict__ istate,
                         int advance_step, const int *__restrict__ sys_of, int batch,
                         const int *__restrict__ gs, const unsigned char *__restrict__ frz) {
  if (gated_off(gs, 0)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[6] = {0, 0, 0, 0, 0, 0};
  int sy = -1;
  if (i < n) {
    sy = sys_of[i];
    double r = 1. / mass[i];
    // freeze_atom closes the force level: the atom keeps no velocity and
    // no force, so the kick below leaves it at rest
    const bool frozen = frz && frz[i];
    for (int d = 0; d < 3; d++) {
      int x = d * n + i;
      if (rm_l) fxl[x] *= r;
      if (rm_s) fxs[x] *= r;
      if (frozen) {
        if (level == 1) fxl[x] = 0.;
        fxs[x] = 0.;
        vel[x] = 0.;
      }
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
  P.nchain = c->nchain;
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

// cross bonds, torsions, 1-4 pairs (global atom indices, CM3D's order within
// each system, systems in batch order) and their parameters, and the frozen
// atoms, as read from the system descriptions
struct IntraHost {
  std::vector<int4> bx, tor, o14;        // {i, j, k, -} / {i, j, k, l} / {i, j, type, -}
  std::vector<double4> bx_par;
  std::vector<int2> tor_par;             // {form, row}
  std::vector<double2> tor_h;
  std::vector<double> tor_v;
  std::vector<double4> o14_rng;
  std::vector<double> o14_se, o14_v, o14_dv;
  std::vector<int2> o14_tab;
  std::vector<unsigned char> frz;
  bool any_frz = false;
};

static int collect_intra(Ctx *c, const cm3d_nb_system *systems, int nsys, IntraHost &ih) {
  ih.frz.assign((size_t)c->n, 0);
  for (int sy = 0; sy < nsys; sy++) {
    const cm3d_nb_system *s = systems + sy;
    const int a0 = c->h_sp[sy].a0, ns = s->natoms;
    auto atom_ok = [&](int i) { return i >= 0 && i < ns; };
    // every array a nonzero count refers to must be there
    const bool missing =
        (s->nbondx > 0 && (!s->ibondx || !s->jbondx || !s->kbondx || !s->idxbondx || !s->eq1bondx ||
                           !s->eq2bondx || !s->fkbondx)) ||
        (s->ntors > 0 && (!s->itors || !s->jtors || !s->ktors || !s->ltors || !s->idxtors || !s->tors_ind_pot ||
                          !s->tors_ind_pot_num || (s->ntors_harm > 0 && (!s->eqtors || !s->fktors)) ||
                          (s->ntors_series > 0 && !s->vphi))) ||
        (s->n14 > 0 && (!s->i14 || !s->j14 || !s->i14dx || !s->r14min2 || !s->r14max2 || !s->dx214tab ||
                        !s->v14tab || !s->dv14tab)) ||
        (s->nfreeze > 0 && !s->ifreeze);
    if (missing) {
      set_error("system %d: a cross-bond, torsion, 1-4 or frozen-atom array is NULL while its count is not 0", sy);
      return CM3D_NB_ERR_ARG;
    }
    for (int b = 0; b < s->nbondx; b++) {
      const int t = s->idxbondx[b];
      if (t < 0 || t >= s->nbondx_types || !atom_ok(s->ibondx[b]) || !atom_ok(s->jbondx[b]) ||
          !atom_ok(s->kbondx[b])) {
        set_error("system %d cross bond %d: type or atom index out of range", sy, b);
        return CM3D_NB_ERR_ARG;
      }
      ih.bx.push_back(make_int4(a0 + s->ibondx[b], a0 + s->jbondx[b], a0 + s->kbondx[b], 0));
      ih.bx_par.push_back(make_double4(s->eq1bondx[t], s->eq2bondx[t], s->fkbondx[t], 0.));
    }
    const int h0 = (int)ih.tor_h.size(), v0 = (int)(ih.tor_v.size() / CM3D_NB_MAXPOWER_TORS);
    if (s->ntors > 0) {
      for (int k = 0; k < s->ntors_harm; k++) ih.tor_h.push_back(make_double2(s->eqtors[k], s->fktors[k]));
      for (int k = 0; k < s->ntors_series * CM3D_NB_MAXPOWER_TORS; k++) ih.tor_v.push_back(s->vphi[k]);
    }
    for (int t = 0; t < s->ntors; t++) {
      const int ty = s->idxtors[t];
      if (ty < 0 || ty >= s->ntors_types || !atom_ok(s->itors[t]) || !atom_ok(s->jtors[t]) ||
          !atom_ok(s->ktors[t]) || !atom_ok(s->ltors[t])) {
        set_error("system %d torsion %d: type or atom index out of range", sy, t);
        return CM3D_NB_ERR_ARG;
      }
      const int form = s->tors_ind_pot[ty], row = s->tors_ind_pot_num[ty];
      int2 par;
      if (form == 0 && row >= 0 && row < s->ntors_harm) {
        par = make_int2(0, h0 + row);
      } else if (form == 1 && row >= 0 && row < s->ntors_series) {
        par = make_int2(1, v0 + row);
      } else if (form == 2) {
        // CM3D's getvtors has no break after this case and stops in its
        // default branch (md_ftors.c:398-423), so no run uses it
        set_error("system %d torsion type %d: the cosine series with phases (ind_pot 2) is not supported", sy, ty);
        return CM3D_NB_ERR_ARG;
      } else {
        set_error("system %d torsion type %d: form %d / row %d out of range", sy, ty, form, row);
        return CM3D_NB_ERR_ARG;
      }
      ih.tor.push_back(make_int4(a0 + s->itors[t], a0 + s->jtors[t], a0 + s->ktors[t], a0 + s->ltors[t]));
      ih.tor_par.push_back(par);
    }
    const int o0 = (int)ih.o14_rng.size();
    if (s->n14 > 0) {
      if (s->n14table < 4) {
        set_error("system %d: 1-4 tables of %d knots", sy, s->n14table);
        return CM3D_NB_ERR_ARG;
      }
      for (int t = 0; t < s->n14_types; t++) {
        ih.o14_rng.push_back(make_double4(s->r14min2[t], s->r14max2[t], s->dx214tab[t], s->scale_onefour));
        ih.o14_se.push_back(s->scale_onefour_e);
        ih.o14_tab.push_back(make_int2((int)ih.o14_v.size(), s->n14table));
        const size_t k0 = (size_t)t * s->n14table;
        ih.o14_v.insert(ih.o14_v.end(), s->v14tab + k0, s->v14tab + k0 + s->n14table);
        ih.o14_dv.insert(ih.o14_dv.end(), s->dv14tab + k0, s->dv14tab + k0 + s->n14table);
      }
    }
    for (int k = 0; k < s->n14; k++) {
      const int ty = s->i14dx[k];
      if (ty < 0 || ty >= s->n14_types || !atom_ok(s->i14[k]) || !atom_ok(s->j14[k])) {
        set_error("system %d 1-4 pair %d: type or atom index out of range", sy, k);
        return CM3D_NB_ERR_ARG;
      }
      ih.o14.push_back(make_int4(a0 + s->i14[k], a0 + s->j14[k], o0 + ty, 0));
    }
    for (int f = 0; f < s->nfreeze; f++) {
      if (!atom_ok(s->ifreeze[f])) {
        set_error("system %d frozen atom %d out of range", sy, s->ifreeze[f]);
        return CM3D_NB_ERR_ARG;
      }
      ih.frz[(size_t)(a0 + s->ifreeze[f])] = 1;
      ih.any_frz = true;
    }
  }
  return CM3D_NB_OK;
}

// group the intramolecular terms (CM3D's order kept inside a group) and copy
// them, with their parameters and the frozen-atom flags, to one device buffer
static int upload_intra(Ctx *c, const IntraHost &ih, const std::vector<int> &gid, int ng) {
  c->has_tors_level = !ih.tor.empty() || !ih.o14.empty();
  c->has_intra_x = c->has_tors_level || !ih.bx.empty();
  if (!c->has_intra_x && !ih.any_frz) return CM3D_NB_OK;
  std::vector<char> h;
  auto add = [&](const void *p, size_t bytes) {
    size_t off = (h.size() + 15) & ~(size_t)15;
    h.resize(off + (bytes > 0 ? bytes : 16));
    if (bytes) memcpy(&h[off], p, bytes);
    return off;
  };
  // a term goes to the group of its first atom; the offsets are per group
  auto group_terms = [&](const std::vector<int4> &terms, std::vector<int> &off, std::vector<int> &order) {
    off.assign((size_t)ng + 1, 0);
    for (const int4 &t : terms) off[gid[t.x] + 1]++;
    for (int g = 0; g < ng; g++) off[g + 1] += off[g];
    std::vector<int> cur(off.begin(), off.end() - 1);
    order.assign(terms.size(), 0);
    for (size_t k = 0; k < terms.size(); k++) order[cur[gid[terms[k].x]]++] = (int)k;
  };
  size_t o_bx_off = 0, o_bx = 0, o_bxp = 0, o_tor_off = 0, o_tor = 0, o_torp = 0, o_th = 0, o_tv = 0;
  size_t o_o14_off = 0, o_o14 = 0, o_rng = 0, o_se = 0, o_tab = 0, o_v = 0, o_dv = 0, o_frz = 0;
  if (c->has_intra_x) {
    std::vector<int> off, order;
    group_terms(ih.bx, off, order);
    std::vector<int4> bx(order.size());
    std::vector<double4> bxp(order.size());
    for (size_t k = 0; k < order.size(); k++) {
      bx[k] = ih.bx[order[k]];
      bxp[k] = ih.bx_par[order[k]];
    }
    o_bx_off = add(off.data(), sizeof(int) * off.size());
    o_bx = add(bx.data(), sizeof(int4) * bx.size());
    o_bxp = add(bxp.data(), sizeof(double4) * bxp.size());
    group_terms(ih.tor, off, order);
    std::vector<int4> tor(order.size());
    std::vector<int2> torp(order.size());
    for (size_t k = 0; k < order.size(); k++) {
      tor[k] = ih.tor[order[k]];
      torp[k] = ih.tor_par[order[k]];
    }
    o_tor_off = add(off.data(), sizeof(int) * off.size());
    o_tor = add(tor.data(), sizeof(int4) * tor.size());
    o_torp = add(torp.data(), sizeof(int2) * torp.size());
    o_th = add(ih.tor_h.data(), sizeof(double2) * ih.tor_h.size());
    o_tv = add(ih.tor_v.data(), sizeof(double) * ih.tor_v.size());
    group_terms(ih.o14, off, order);
    std::vector<int4> o14(order.size());
    for (size_t k = 0; k < order.size(); k++) o14[k] = ih.o14[order[k]];
    o_o14_off = add(off.data(), sizeof(int) * off.size());
    o_o14 = add(o14.data(), sizeof(int4) * o14.size());
    o_rng = add(ih.o14_rng.data(), sizeof(double4) * ih.o14_rng.size());
    o_se = add(ih.o14_se.data(), sizeof(double) * ih.o14_se.size());
    o_tab = add(ih.o14_tab.data(), sizeof(int2) * ih.o14_tab.size());
    o_v = add(ih.o14_v.data(), sizeof(double) * ih.o14_v.size());
    o_dv = add(ih.o14_dv.data(), sizeof(double) * ih.o14_dv.size());
  }
  if (ih.any_frz) o_frz = add(ih.frz.data(), ih.frz.size());
  CK(cudaMalloc(&c->intra_buf, h.size()));
  CK(cudaMemcpy(c->intra_buf, h.data(), h.size(), cudaMemcpyHostToDevice));
  const char *b = reinterpret_cast<const char *>(c->intra_buf);
  IntraDev &X = c->intra;
  if (c->has_intra_x) {
    X.bx_off = reinterpret_cast<const int *>(b + o_bx_off);
    X.bx_ijk = reinterpret_cast<const int4 *>(b + o_bx);
    X.bx_par = reinterpret_cast<const double4 *>(b + o_bxp);
    X.tor_off = reinterpret_cast<const int *>(b + o_tor_off);
    X.tor_ijkl = reinterpret_cast<const int4 *>(b + o_tor);
    X.tor_par = reinterpret_cast<const int2 *>(b + o_torp);
    X.tor_h = reinterpret_cast<const double2 *>(b + o_th);
    X.tor_v = reinterpret_cast<const double *>(b + o_tv);
    X.o14_off = reinterpret_cast<const int *>(b + o_o14_off);
    X.o14_ij = reinterpret_cast<const int4 *>(b + o_o14);
    X.o14_rng = reinterpret_cast<const double4 *>(b + o_rng);
    X.o14_se = reinterpret_cast<const double *>(b + o_se);
    X.o14_tab = reinterpret_cast<const int2 *>(b + o_tab);
    X.o14_v = reinterpret_cast<const double *>(b + o_v);
    X.o14_dv = reinterpret_cast<const double *>(b + o_dv);
  }
  if (ih.any_frz) X.frz = reinterpret_cast<const unsigned char *>(b + o_frz);
  return CM3D_NB_OK;
}

// Nose-Hoover chains of every system, thermostats numbered across the batch
// (system order), with their state as CM3D holds it after samveta
static int nvt_setup(Ctx *c, const cm3d_nb_system *systems, int nsys) {
  if (systems[0].iensemble != 1) return CM3D_NB_OK;
  const int nch = systems[0].nchain;
  int nt = 0;
  for (int sy = 0; sy < nsys; sy++) nt += systems[sy].ntherm;
  const size_t tc = (size_t)nt * nch;
  std::vector<double> h(5 * tc + (size_t)nt, 0.0);
  std::vector<int> thm((size_t)c->n, -1);
  int t0 = 0;
  c->therm0.assign((size_t)nsys + 1, 0);
  for (int sy = 0; sy < nsys; sy++) {
    const cm3d_nb_system *s = systems + sy;
    const size_t o = (size_t)t0 * nch, k = (size_t)s->ntherm * nch;
    c->therm0[(size_t)sy] = t0;
    std::copy(s->mnh, s->mnh + k, h.begin() + o);
    std::copy(s->gkt, s->gkt + k, h.begin() + tc + o);
    std::copy(s->nhc_eta, s->nhc_eta + k, h.begin() + 2 * tc + o);
    std::copy(s->nhc_veta, s->nhc_veta + k, h.begin() + 3 * tc + o);
    for (int i = 0; i < s->natoms; i++) {
      const int j = s->ithm[i];
      if (j >= s->ntherm) {
        set_error("system %d atom %d: thermostat %d of %d", sy, i, j, s->ntherm);
        return CM3D_NB_ERR_ARG;
      }
      thm[(size_t)(c->h_sp[sy].a0 + i)] = j >= 0 ? t0 + j : -1;
    }
    t0 += s->ntherm;
  }
  c->therm0[(size_t)nsys] = t0;
  c->ntherm = nt;
  c->nchain = nch;
  CK(cudaMalloc(&c->nhc, sizeof(double) * h.size()));
  CK(cudaMemcpy(c->nhc, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&c->ithm, sizeof(int) * thm.size()));
  CK(cudaMemcpy(c->ithm, thm.data(), sizeof(int) * thm.size(), cudaMemcpyHostToDevice));
  // the thermostats' atoms in thermostat order (atom order inside one) and
  // their chunks of at most NVT_CHUNK atoms
  constexpr int NVT_CHUNK = 1024;
  std::vector<std::vector<int>> by(nt);
  for (int i = 0; i < c->n; i++)
    if (thm[(size_t)i] >= 0) by[(size_t)thm[(size_t)i]].push_back(i);
  std::vector<int> atoms, choff(1, 0);
  std::vector<int2> chunks;
  for (int j = 0; j < nt; j++) {
    const int a0 = (int)atoms.size();
    atoms.insert(atoms.end(), by[(size_t)j].begin(), by[(size_t)j].end());
    for (int k = a0; k < (int)atoms.size(); k += NVT_CHUNK)
      chunks.push_back(make_int2(k, std::min((int)atoms.size(), k + NVT_CHUNK)));
    choff.push_back((int)chunks.size());
  }
  c->nth_chunks = (int)chunks.size();
  CK(cudaMalloc(&c->nvt_kin, sizeof(double) * (size_t)c->n));
  CK(cudaMemset(c->nvt_kin, 0, sizeof(double) * (size_t)c->n));
  CK(cudaMalloc(&c->th_atoms, sizeof(int) * std::max<size_t>(atoms.size(), 1)));
  if (!atoms.empty()) CK(cudaMemcpy(c->th_atoms, atoms.data(), sizeof(int) * atoms.size(), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&c->th_chunk, sizeof(int2) * std::max<size_t>(chunks.size(), 1)));
  if (!chunks.empty())
    CK(cudaMemcpy(c->th_chunk, chunks.data(), sizeof(int2) * chunks.size(), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&c->nvt_chsum, sizeof(double) * std::max<size_t>(chunks.size(), 1)));
  CK(cudaMalloc(&c->th_choff, sizeof(int) * choff.size()));
  CK(cudaMemcpy(c->th_choff, choff.data(), sizeof(int) * choff.size(), cudaMemcpyHostToDevice));
  return CM3D_NB_OK;
}

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
  IntraHost ih;
  int rc;
  if ((rc = collect_intra(c, systems, nsys, ih))) return rc;
  const int nb = (int)mb.size(), ne = (int)me.size(), nc = (int)mc.size();
  UF uf(n);
  for (int b = 0; b < nb; b++) uf.u(mb[b].x, mb[b].y);
  for (int b = 0; b < ne; b++) {
    uf.u(me[b].x, me[b].y);
    uf.u(me[b].y, me[b].z);
  }
  for (int b = 0; b < nc; b++) uf.u(mc[b].x, mc[b].y);
  for (const int4 &t : ih.bx) {
    uf.u(t.x, t.y);
    uf.u(t.y, t.z);
  }
  for (const int4 &t : ih.tor) {
    uf.u(t.x, t.y);
    uf.u(t.y, t.z);
    uf.u(t.z, t.w);
  }
  for (const int4 &t : ih.o14) uf.u(t.x, t.y);
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
  // the groups k_group_init has work for
  {
    std::vector<int> work;
    for (int g = 0; g < ng; g++)
      if (coff[g + 1] > coff[g] || boff[g + 1] > boff[g] || eoff[g + 1] > eoff[g]) work.push_back(g);
    c->ngwork = (int)work.size();
    CK(cudaMalloc(&c->grp_work, sizeof(int) * (work.empty() ? 1 : work.size())));
    if (!work.empty()) CK(cudaMemcpy(c->grp_work, work.data(), sizeof(int) * work.size(), cudaMemcpyHostToDevice));
  }
  if ((rc = upload_intra(c, ih, gid, ng))) return rc;
  return nvt_setup(c, systems, nsys);
}

int run_bonded(Ctx *c) {
  StepP P = step_params(c);
  const int B = 128;
  k_bonded<<<grid_for(c->ngroups, B), B, 0, c->st>>>(P, c->grp_atom_off, c->grp_atoms, c->pos, c->mass, c->vel,
                                                     c->fxa, c->grp_bond_off, c->bond_ij, c->bond_p,
                                                     c->grp_bend_off, c->bend_ijk, c->bend_p, c->intra);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

// force(3): the torsion level (torsions + 1-4 pairs) into fxr; with neither
// in the context fxr is zero and only frozen atoms need their velocity cleared
int run_tors_level(Ctx *c) {
  if (!c->has_tors_level && !c->intra.frz) {
    CK(cudaMemsetAsync(c->fxr, 0, sizeof(double) * 3 * (size_t)c->n, c->st));
    return CM3D_NB_OK;
  }
  StepP P = step_params(c);
  const int B = 128;
  if (!c->has_tors_level) CK(cudaMemsetAsync(c->fxr, 0, sizeof(double) * 3 * (size_t)c->n, c->st));
  k_tors_level<<<grid_for(c->ngroups, B), B, 0, c->st>>>(P, c->grp_atom_off, c->grp_atoms, c->pos, c->q, c->mass,
                                                         c->vel, c->fxr, c->intra, c->stat);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

int group_init(Ctx *c, bool zero_fxs) {
  StepP P = step_params(c);
  const int B = 128;
  cudaEvent_t e0;
  tbegin(c, 3, &e0);
  // the force arrays start from zero (a halted graph step zeroes them too:
  // the host-driven path that finishes it computes them again from here)
  CK(cudaMemsetAsync(c->fxl, 0, sizeof(double) * 3 * (size_t)c->n, c->st));
  if (zero_fxs) CK(cudaMemsetAsync(c->fxs, 0, sizeof(double) * 3 * (size_t)c->n, c->st));
  if (c->ngwork > 0) {
    k_group_init<<<grid_for(c->ngwork, B), B, 0, c->st>>>(P, c->grp_work, c->ngwork, c->grp_atom_off, c->grp_atoms,
                                                          c->pos, c->q, c->fxl, c->fxs, c->grp_ecorr_off,
                                                          c->ecorr_ij, c->grp_bond_off, c->bond_ij, c->bond_p,
                                                          c->grp_bend_off, c->bend_ijk, c->bend_p, c->acc, c->sp,
                                                          c->sys_of, c->gate);
    c->launches++;
  }
  if (c->has_intra_x) {
    k_intra_energy<<<grid_for(c->ngroups, B), B, 0, c->st>>>(P, c->grp_atom_off, c->grp_atoms, c->pos, c->q,
                                                             c->intra, c->acc, c->sys_of, c->gate);
    c->launches++;
  }
  tend(c, 3, e0);
  CKL(c);
  return CM3D_NB_OK;
}

int finish_level1(Ctx *c, double dter, double dter1, bool kick) {
  const int B = 256;
  bool rs = c->need_short || c->nres_lrf > 1;
  k_finish<<<grid_for(c->n, B), B, 0, c->st>>>(c->n, 1, kick ? 1 : 0, 1, rs ? 1 : 0, dter, dter1, c->mass, c->fxl,
                                               c->fxs, c->vel, c->acc, c->istate, kick ? 1 : 0, c->sys_of,
                                               c->nsys > 1, c->gate, c->intra.frz);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

static int finish_level0(Ctx *c, double dts2, bool kick) {
  k_finish<<<grid_for(c->n, 256), 256, 0, c->st>>>(c->n, 0, kick ? 1 : 0, 0, 1, 0, dts2, c->mass, c->fxl, c->fxs,
                                                   c->vel, c->acc, c->istate, 0, c->sys_of, c->nsys > 1, c->gate,
                                                   c->intra.frz);
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

// force(iflg) of md_fcntr.c:44-134 (levels 0-3)
int run_force(Ctx *c, int iflg) {
  int rc;
  if (iflg == 2) return run_bonded(c);
  if (iflg == 3) return run_tors_level(c);
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
// force(1) + kick on the last level, force(0) + kick otherwise.  ks_forked:
// the accumulators were zeroed and the k-space runs on the side stream
// already (kspace_fork), joined here after the pair forces.
static int close_level(Ctx *c, int intr, bool ks_forked = false) {
  int rc;
  StepP P = step_params(c);
  if (intr == c->nres_lrf - 1) {
    if (!ks_forked && (rc = zero_acc(c))) return rc;
    if ((rc = group_init(c, P.use_fxs))) return rc;
    if ((rc = pair_forces(c, 1, 3))) return rc;
    if ((rc = ks_forked ? kspace_join(c) : kspace_forces(c))) return rc;
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
  if (c->ntherm > 0) {
    // NVT: four launches per inner substep (k_nvt_a, k_nvt_ksum, k_nvt_chain, k_nvt_c)
    const size_t tc = (size_t)c->ntherm * c->nchain;
    double *veta = c->nhc + 3 * tc;
    for (int inrra = 0; inrra < c->nres_tors; inrra++)
      for (int intra = 0; intra < c->nres_intra; intra++) {
        k_nvt_a<<<grid_for(c->ngroups, B), B, 0, c->st>>>(P, intr, inrra == 0 && intra == 0, intra == 0,
                                                          c->grp_atom_off, c->grp_atoms, c->pos, c->vel, c->mass,
                                                          c->fxl, c->fxs, c->fxa, c->fxr, c->ithm, veta, c->nvt_kin,
                                                          c->intra, c->istate, c->gate);
        k_nvt_ksum<<<grid_for(32LL * c->nth_chunks, 256), 256, 0, c->st>>>(c->nth_chunks, c->th_chunk, c->th_atoms,
                                                                          c->nvt_kin, c->nvt_chsum, c->gate);
        k_nvt_chain<<<grid_for(c->ntherm, 64), 64, 0, c->st>>>(c->ntherm, c->nchain, P.dta2, c->nhc, c->nvt_chsum,
                                                               c->th_choff,
                                                               c->gate);
        k_nvt_c<<<grid_for(c->ngroups, B), B, 0, c->st>>>(
            P, intra == c->nres_intra - 1, inrra == c->nres_tors - 1 && intra == c->nres_intra - 1,
            c->grp_atom_off, c->grp_atoms, c->pos, c->vel, c->mass, c->q, c->fxa, c->fxr, c->dxn,
            c->grp_bond_off, c->bond_ij, c->bond_p, c->grp_bend_off, c->bend_ijk, c->bend_p, c->ithm, veta,
            c->sp, c->sys_of, c->sreb, c->istate, c->intra, c->stat, c->gate);
        c->launches += 4;
      }
  } else {
    auto inner = c->has_intra_x || c->intra.frz ? k_inner<true> : k_inner<false>;
    inner<<<grid_for(c->ngroups, B), B, 0, c->st>>>(P, intr, c->grp_atom_off, c->grp_atoms, c->pos, c->vel,
                                                      c->mass, c->fxl, c->fxs, c->fxa, c->dxn, c->grp_bond_off,
                                                      c->bond_ij, c->bond_p, c->grp_bend_off, c->bend_ijk,
                                                      c->bend_p, c->sp, c->sys_of, c->sreb, c->istate, c->gate,
                                                      c->intra, c->q, c->fxr, c->stat);
    c->launches++;
  }
  tend(c, 3, e0);
  CKL(c);
  if ((rc = reset_positions(c))) return rc;
  if (intr == c->nres_lrf - 1 && c->ho_pos) {
    // the step's positions are final: their copy to the registered host
    // buffer runs on a third stream beside the rest of the step (joined at
    // the step's end)
    CK(cudaEventRecord(c->ev_f3, c->st));
    CK(cudaStreamWaitEvent(c->st3, c->ev_f3, 0));
    CK(cudaMemcpyAsync(c->ho_pos, c->pos, sizeof(double) * 3 * (size_t)c->n, cudaMemcpyDeviceToHost, c->st3));
    CK(cudaEventRecord(c->ev_j3, c->st3));
    c->ho_forked = true;
  }
  // the positions are final for this level: force(1)'s k-space can start on
  // the side stream while the lists are rebuilt and the pair forces run
  const bool fork = intr == c->nres_lrf - 1 && kspace_async_ok(c);
  if (fork) {
    if ((rc = zero_acc(c))) return rc;
    if ((rc = kspace_fork(c))) return rc;
  }
  if (gated) {
    if ((rc = build_lists(c, true, false))) return rc;
  } else {
    CK(cudaMemcpyAsync(c->h_istate, c->istate, sizeof(int) * IS_COUNT, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (c->h_istate[IS_REBUILD]) {
      if ((rc = build_lists(c, false, false))) return rc;
    }
  }
  return close_level(c, intr, fork);
}

static int one_step(Ctx *c, bool gated) {
  for (int intr = 0; intr < c->nres_lrf; intr++) {
    int rc = one_level(c, intr, gated);
    if (rc) return rc;
  }
  return host_outputs_tail(c);
}

static int set_istep(Ctx *c, int istep) {
  c->h_istate[IS_ISTEP] = istep;
  CK(cudaMemcpyAsync(c->istate + IS_ISTEP, c->h_istate + IS_ISTEP, sizeof(int), cudaMemcpyHostToDevice, c->st));
  return CM3D_NB_OK;
}

// the end of a step with registered host outputs: join the positions' copy
// and copy the velocities
int host_outputs_tail(Ctx *c) {
  if (c->ho_forked) {
    CK(cudaStreamWaitEvent(c->st, c->ev_j3, 0));
    c->ho_forked = false;
  }
  if (c->ho_vel)
    CK(cudaMemcpyAsync(c->ho_vel, c->vel, sizeof(double) * 3 * (size_t)c->n, cudaMemcpyDeviceToHost, c->st));
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
    DevLock lock(device_mutex());
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
  if (!c->pending) {
    // eager steps ran here already; their copies to registered host
    // outputs may still be in flight
    if (c->ho_pos || c->ho_vel) CK(cudaStreamSynchronize(c->st));
    return CM3D_NB_OK;
  }
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
  // the halted step copied its positions (final before its list build) and
  // stale velocities: the step's outputs again, complete before returning
  if ((rc = host_outputs_tail(c))) return rc;
  if (c->ho_pos || c->ho_vel) CK(cudaStreamSynchronize(c->st));
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
