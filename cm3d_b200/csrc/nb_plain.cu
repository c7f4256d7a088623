// nb_plain.cu -- the plain FP64 comparator: CM3D's pair kernels one pair per
// thread over CM3D's own half lists, FP64 throughout, atomic force scatter.
//
// Restates force_npol (energy/inter/md_fnopol.c:46-255), force_e
// (energy/inter/finter_e.c:42-233) and ecorr (energy/inter/md_ewald.c:385-453)
// per pair, in CM3D's operation order (this file is compiled with
// -fmad=false), so each pair's force, energy and virial term is bit-identical
// to CM3D's; only the order in which the terms are summed differs.
#include "nb_common.cuh"

namespace cm3d {

struct PlainP {
  double h[9], hi[9];
  int ntypes, ntable, iflg, need_s;
  double dx2coul, rmins_coul2, rmaxl_coul2, tablast;
};

// 3-point interpolation of md_fnopol.c:148, CM3D's grouping
__device__ __forceinline__ double interp_ref(const double *t, int k, double p) {
  double fm1 = t[k - 1], f0 = t[k], f1 = t[k + 1];
  return f0 + .5 * p * (f1 - fm1 + p * (fm1 - 2. * f0 + f1));
}

// LJ over a half list (t at iflg 1, s at iflg 0)
__global__ void k_lj_plain(const long long *__restrict__ npd, const int2 *__restrict__ lst, PlainP P, int n,
                           const double *__restrict__ pos, const int *__restrict__ itype,
                           const int *__restrict__ map, const double *__restrict__ icut,
                           const double *__restrict__ dvtab, const double *__restrict__ vtab,
                           const double *__restrict__ switchs, double *__restrict__ fl,
                           double *__restrict__ fs, double *__restrict__ acc, long long *__restrict__ stat,
                           const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  // v: spotl spothl sprsl t0 t1 t2 t4 t5 t8
  double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  long long under = 0;
  const long long np = *npd;   // device count: valid after device-side rebuilds
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
       p += (long long)gridDim.x * blockDim.x) {
    int2 pr = lst[p];
    int i = pr.x, j = pr.y;
    double dx = pos[i] - pos[j], dy = pos[n + i] - pos[n + j], dz = pos[2 * n + i] - pos[2 * n + j];
    period_ref(dx, dy, dz, P.h, P.hi);
    int in = map[itype[i] * P.ntypes + itype[j]];
    double dis2 = dx * dx + dy * dy + dz * dz;
    const double *c = icut + 8 * in;
    double rmax2 = P.iflg == 0 ? c[0] : c[2];
    if (!(dis2 < rmax2)) continue;
    double pp = (dis2 - c[1]) * c[6];
    int k = (int)pp;
    if (k < 1) {
      under++;
      k = 1;
      pp = 1.;
    }
    pp = pp - (double)k;
    const size_t base = (size_t)in * P.ntable;
    double f = interp_ref(dvtab + base, k, pp);
    double swv = dis2 > c[3] ? interp_ref(switchs + base, k, pp) : 1.;
    double fx, fy, fz;
    if (P.iflg == 1) {
      v[2] -= dis2 * f;
      v[3] -= dx * dx * f;
      v[4] -= dy * dx * f;
      v[5] -= dz * dx * f;
      v[6] -= dy * dy * f;
      v[7] -= dz * dy * f;
      v[8] -= dz * dz * f;
      fx = dx * f;
      fy = dy * f;
      fz = dz * f;
      double fcc = interp_ref(vtab + base, k, pp);
      v[0] += fcc;
      v[1] += fcc - c[7];
      if (P.need_s) {
        double sx = fx * swv, sy = fy * swv, sz = fz * swv;
        atomicAdd(fs + i, -sx); atomicAdd(fs + n + i, -sy); atomicAdd(fs + 2 * n + i, -sz);
        atomicAdd(fs + j, sx); atomicAdd(fs + n + j, sy); atomicAdd(fs + 2 * n + j, sz);
      }
    } else {
      f *= swv;
      fx = dx * f;
      fy = dy * f;
      fz = dz * f;
    }
    atomicAdd(fl + i, -fx); atomicAdd(fl + n + i, -fy); atomicAdd(fl + 2 * n + i, -fz);
    atomicAdd(fl + j, fx); atomicAdd(fl + n + j, fy); atomicAdd(fl + 2 * n + j, fz);
  }
  if (under) atomicAdd((unsigned long long *)(stat + ST_UNDERFLOW), (unsigned long long)under);
  if (P.iflg == 1) {
    const int slots[9] = {ACC_SPOTL, ACC_SPOTHL, ACC_SPRSL, ACC_SPRSLT + 0, ACC_SPRSLT + 1,
                          ACC_SPRSLT + 2, ACC_SPRSLT + 4, ACC_SPRSLT + 5, ACC_SPRSLT + 8};
    block_acc<9>(v, acc, slots);
  }
}

// real-space Ewald over a half list (te at iflg 1, se at iflg 0); CM3D's
// force_e falls through from level 0 into level 1 (finter_e.c:72-83), so
// both levels use the full cutoff rmaxl_coul2 and the switch never engages
__global__ void k_el_plain(const long long *__restrict__ npd, const int2 *__restrict__ lst, PlainP P, int n,
                           const double *__restrict__ pos, const double *__restrict__ q,
                           const double *__restrict__ dcoultab, const double *__restrict__ coultab,
                           double *__restrict__ fl, double *__restrict__ fs, double *__restrict__ acc,
                           long long *__restrict__ stat, const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  // v: spote spothe sprse t0 t1 t2 t4 t5 t8
  double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  long long under = 0;
  const long long np = *npd;   // device count: valid after device-side rebuilds
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
       p += (long long)gridDim.x * blockDim.x) {
    int2 pr = lst[p];
    int i = pr.x, j = pr.y;
    double dx = pos[i] - pos[j], dy = pos[n + i] - pos[n + j], dz = pos[2 * n + i] - pos[2 * n + j];
    double qij = q[i] * q[j];
    period_ref(dx, dy, dz, P.h, P.hi);
    double dis2 = dx * dx + dy * dy + dz * dz;
    if (!(dis2 < P.rmaxl_coul2)) continue;
    double pp = (dis2 - P.rmins_coul2) * P.dx2coul;
    int k = (int)pp;
    if (k < 1) {
      under++;
      k = 1;
      pp = 1;
    }
    pp = pp - (double)k;
    double f = interp_ref(dcoultab, k, pp);
    double fcc = qij * f;
    double fx = dx * fcc, fy = dy * fcc, fz = dz * fcc;
    if (P.iflg == 1) {
      v[2] -= dis2 * fcc;
      v[3] -= dx * dx * fcc;
      v[4] -= dy * dx * fcc;
      v[5] -= dz * dx * fcc;
      v[6] -= dy * dy * fcc;
      v[7] -= dz * dy * fcc;
      v[8] -= dz * dz * fcc;
      double e = interp_ref(coultab, k, pp);
      v[1] += qij * (e - P.tablast);
      v[0] += qij * e;
      if (P.need_s) {
        atomicAdd(fs + i, -fx); atomicAdd(fs + n + i, -fy); atomicAdd(fs + 2 * n + i, -fz);
        atomicAdd(fs + j, fx); atomicAdd(fs + n + j, fy); atomicAdd(fs + 2 * n + j, fz);
      }
    }
    atomicAdd(fl + i, -fx); atomicAdd(fl + n + i, -fy); atomicAdd(fl + 2 * n + i, -fz);
    atomicAdd(fl + j, fx); atomicAdd(fl + n + j, fy); atomicAdd(fl + 2 * n + j, fz);
  }
  if (under) atomicAdd((unsigned long long *)(stat + ST_UNDERFLOW), (unsigned long long)under);
  if (P.iflg == 1) {
    const int slots[9] = {ACC_SPOTE, ACC_SPOTHE, ACC_SPRSE, ACC_SPRSET + 0, ACC_SPRSET + 1,
                          ACC_SPRSET + 2, ACC_SPRSET + 4, ACC_SPRSET + 5, ACC_SPRSET + 8};
    block_acc<9>(v, acc, slots);
  }
}

// excluded-pair Ewald correction, one pair per thread (no minimum image, as
// in CM3D, md_ewald.c:409-413)
__global__ void k_ecorr_plain(int necorr, const int2 *__restrict__ ij, int n, const double *__restrict__ pos,
                              const double *__restrict__ q, double kappa, double kappa2,
                              double *__restrict__ fl, double *__restrict__ acc) {
  double v[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double sqrt_pi = 1. / sqrt(M_PI);
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < necorr; p += gridDim.x * blockDim.x) {
    int ii = ij[p].x, jj = ij[p].y;
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
    atomicAdd(fl + ii, xd); atomicAdd(fl + n + ii, yd); atomicAdd(fl + 2 * n + ii, zd);
    atomicAdd(fl + jj, -xd); atomicAdd(fl + n + jj, -yd); atomicAdd(fl + 2 * n + jj, -zd);
  }
  const int slots[8] = {ACC_POT_ECORR, ACC_PRS_ECORR, ACC_PRS_ECORRT + 0, ACC_PRS_ECORRT + 1,
                        ACC_PRS_ECORRT + 2, ACC_PRS_ECORRT + 4, ACC_PRS_ECORRT + 5, ACC_PRS_ECORRT + 8};
  double w[8] = {v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]};
  block_acc<8>(w, acc, slots);
}

static PlainP plain_params(Ctx *c, int iflg) {
  PlainP P;
  for (int k = 0; k < 9; k++) {
    P.h[k] = c->hmat[k];
    P.hi[k] = c->hmati[k];
  }
  P.ntypes = c->ntypes;
  P.ntable = c->ntable;
  P.iflg = iflg;
  P.need_s = (iflg == 1) && (c->need_short || c->nres_lrf > 1);
  P.dx2coul = c->dx2coul;
  P.rmins_coul2 = c->rmins_coul2;
  P.rmaxl_coul2 = c->rmaxl_coul2;
  P.tablast = 0;
  return P;
}

// which: 0 LJ, 1 elec.  Accumulates raw forces into fxl (+fxs) for iflg 1,
// into fxs for iflg 0.
int plain_pairs(Ctx *c, int iflg, int which) {
  PlainP P = plain_params(c, iflg);
  double *fl = iflg == 1 ? c->fxl : c->fxs;
  const int B = 256;
  int list = which == 0 ? (iflg == 1 ? LT_T : LT_S) : (iflg == 1 ? LT_TE : LT_SE);
  // the grid is sized from the host's latest count (grid-stride loop); the
  // kernel reads the exact count from the device, which a device-side
  // rebuild inside a CUDA graph may have changed
  long long np = c->hcount[list] > 0 ? c->hcount[list] : 1;
  int grid = grid_for(np, B);
  if (grid < c->num_sms * 8) grid = c->num_sms * 8;
  if (grid > c->num_sms * 16) grid = c->num_sms * 16;
  const long long *npd = c->ltot + list;
  cudaEvent_t e0;
  tbegin(c, 0, &e0);
  if (which == 0) {
    k_lj_plain<<<grid, B, 0, c->st>>>(npd, c->lst[list], P, c->n, c->pos, c->itype, c->map, c->icut, c->dvtab,
                                      c->vtab, c->switchs, fl, c->fxs, c->acc, c->stat, c->gate);
  } else {
    if (c->ncharge == 0) return CM3D_NB_OK;
    P.tablast = c->tablast_e;
    k_el_plain<<<grid, B, 0, c->st>>>(npd, c->lst[list], P, c->n, c->pos, c->q, c->dcoultab, c->coultab, fl,
                                      c->fxs, c->acc, c->stat, c->gate);
  }
  c->launches++;
  tend(c, 0, e0);
  CKL(c);
  return CM3D_NB_OK;
}

int plain_ecorr(Ctx *c, const int2 *ij) {
  if (c->necorr == 0) return CM3D_NB_OK;
  const int B = 256;
  k_ecorr_plain<<<grid_for(c->necorr, B), B, 0, c->st>>>(c->necorr, ij, c->n, c->pos, c->q, c->kappa, c->kappa2,
                                                         c->fxl, c->acc);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

}  // namespace cm3d
