// nb_capi.cu -- the extern "C" entry points of include/cm3d_nb.h.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "nb_common.cuh"

namespace cm3d {

static thread_local char g_err[1024] = "";

std::recursive_mutex &device_mutex() {
  static std::recursive_mutex mu;
  return mu;
}

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}

int cuda_fail(cudaError_t e, const char *what) {
  set_error("CUDA error in %s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
  if (e == cudaErrorMemoryAllocation) return CM3D_NB_ERR_NOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return CM3D_NB_ERR_NODEV;
  return CM3D_NB_ERR_CUDA;
}

void tbegin(Ctx *c, int cls, cudaEvent_t *e0) {
  *e0 = nullptr;
  if (cls == 4 ? !c->timing.steps : !c->timing.on) return;
  cudaEvent_t a, b;
  if (c->timing.pool.size() >= 1) {
    a = c->timing.pool.back().first;
    b = c->timing.pool.back().second;
    c->timing.pool.pop_back();
  } else {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  cudaEventRecord(a, c->st);
  c->timing.pending[cls].push_back({a, b});
  *e0 = a;
}

void tend(Ctx *c, int cls, cudaEvent_t e0) {
  if (!e0) return;
  cudaEventRecord(c->timing.pending[cls].back().second, c->st);
  c->timing.launches[cls]++;
}

static void collect_timing(Ctx *c) {
  cudaStreamSynchronize(c->st);
  for (int k = 0; k < NTCLS; k++) {
    for (auto &pr : c->timing.pending[k]) {
      float ms = 0;
      cudaEventElapsedTime(&ms, pr.first, pr.second);
      c->timing.ms[k] += ms;
      c->timing.pool.push_back(pr);
    }
    c->timing.pending[k].clear();
  }
}

template <typename T>
static int upload(T **dst, const T *src, size_t count) {
  size_t bytes = sizeof(T) * (count > 0 ? count : 1);
  CK(cudaMalloc(dst, bytes));
  if (src && count) CK(cudaMemcpy(*dst, src, sizeof(T) * count, cudaMemcpyHostToDevice));
  else CK(cudaMemset(*dst, 0, bytes));
  return CM3D_NB_OK;
}

static void destroy(Ctx *c) {
  if (!c) return;
  cudaSetDevice(c->dev);
  if (c->graph) cudaGraphExecDestroy(c->graph);
  void *ptrs[] = {c->pos, c->vel, c->fxl, c->fxs, c->fxa, c->mass, c->q, c->dxn, c->snap, c->itype, c->map,
                  c->vtab, c->dvtab, c->switchs, c->icut, c->coultab, c->dcoultab, c->switchse, c->excl_off,
                  c->excl_idx, c->cexcl_off, c->cexcl_idx, c->ftab_lj, c->ftab_el, c->fcut, c->rows, c->row_k0,
                  c->sk, c->spart, c->akf, c->akd, c->kfrac, c->kposd, c->icharge, c->ka_d, c->kb_d, c->kc_d,
                  c->ecorr_pairs, c->grp_atom_off, c->grp_atoms, c->grp_bond_off, c->grp_bend_off,
                  c->grp_ecorr_off, c->bond_ij, c->bond_p, c->bend_ijk, c->bend_p, c->ecorr_ij, c->cell_of,
                  c->cell_start, c->cell_cursor, c->cell_atoms, c->rank, c->cnt, c->off, c->ltot, c->lst[0],
                  c->lst[1], c->lst[2], c->lst[3], c->nbr, c->xq, c->epart, c->styp, c->shift, c->corner,
                  c->cimg, c->nlen, c->acc,
                  c->stat, c->istate, c->sp, c->sys_of, c->cell_sys, c->sreb, c->slast, c->sstat,
                  c->ktile_sys, c->ftile_sys, c->k_sys, c->kf_part, c->ered, c->ered_done, c->sys_items, c->ftab_lj2, c->rb_scan,
                  c->fxr, c->intra_buf, c->ithm, c->nhc, c->cwl, c->cwn, c->cw_tf, c->cw_tg, c->cw_tl,
                  c->cw_part, c->nvt_kin, c->nvt_chsum, c->th_atoms, c->th_choff, c->th_chunk,
                  c->cw_sys, c->cw_sitems, c->cw_items, c->cw_gidx, c->cw_scan, c->grp_work};
  cw_destroy(c);
  for (void *p : ptrs)
    if (p) cudaFree(p);
  void *hp[] = {c->h_acc, c->h_stat, c->h_istate, c->h_ltot, c->h_sstat};
  for (void *p : hp)
    if (p) cudaFreeHost(p);
  for (int k = 0; k < NTCLS; k++)
    for (auto &pr : c->timing.pending[k]) {
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
  for (auto &pr : c->timing.pool) {
    cudaEventDestroy(pr.first);
    cudaEventDestroy(pr.second);
  }
  if (c->step_ev) cudaEventDestroy(c->step_ev);
  if (c->st) cudaStreamDestroy(c->st);
  if (c->st2) cudaStreamDestroy(c->st2);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->st3) cudaStreamDestroy(c->st3);
  if (c->ev_f3) cudaEventDestroy(c->ev_f3);
  if (c->ev_j3) cudaEventDestroy(c->ev_j3);
  delete c;
}

// One context over `nsys` systems (a batch; one system is a batch of one).
// The systems' atoms are concatenated in order; every per-system parameter
// goes to SysP / SysH.  Batches need the mixed engine and the same ntable,
// time step and RESPA levels in every system.
// H^-1 and 1/det H of a system's box into its host and kernel parameters
static void box_params(SysP &P, SysH &H) {
  const double *h = H.hmat;
  double *hi = H.hmati;
  double rvol = 1. / (h[0] * (h[4] * h[8] - h[5] * h[7]) + h[1] * (h[5] * h[6] - h[3] * h[8]) +
                      h[2] * (h[3] * h[7] - h[4] * h[6]));
  hi[0] = (h[4] * h[8] - h[5] * h[7]) * rvol;
  hi[1] = (h[2] * h[7] - h[1] * h[8]) * rvol;
  hi[2] = (h[1] * h[5] - h[2] * h[4]) * rvol;
  hi[3] = (h[5] * h[6] - h[3] * h[8]) * rvol;
  hi[4] = (h[0] * h[8] - h[2] * h[6]) * rvol;
  hi[5] = (h[2] * h[3] - h[0] * h[5]) * rvol;
  hi[6] = (h[3] * h[7] - h[4] * h[6]) * rvol;
  hi[7] = (h[1] * h[6] - h[0] * h[7]) * rvol;
  hi[8] = (h[0] * h[4] - h[1] * h[3]) * rvol;
  P.rvol = rvol;
  for (int k = 0; k < 9; k++) {
    P.h[k] = H.hmat[k];
    P.hi[k] = H.hmati[k];
    P.hF[k] = (float)H.hmat[k];
    P.hiF[k] = (float)H.hmati[k];
  }
}

// width of the box along each direction (1 / |row d of H^-1|)
static double box_width(const SysH &H, int d) {
  return 1.0 / sqrt(H.hmati[3 * d] * H.hmati[3 * d] + H.hmati[3 * d + 1] * H.hmati[3 * d + 1] +
                    H.hmati[3 * d + 2] * H.hmati[3 * d + 2]);
}

// boxes narrower than two list radii need the on-the-fly minimum image (for
// the pairs near the image boundary, see near_s)
static void box_widths(SysP &P, const SysH &H) {
  P.smallbox = 0;
  for (int d = 0; d < 3; d++) {
    const double w = box_width(H, d);
    if (w < 2.0 * H.rlist) P.smallbox = 1;
    P.near_s[d] = 0.5 - 1.01 * H.skin / w - 1e-6;
  }
}

static int create(const cm3d_nb_system *systems, int nsys, const cm3d_nb_options *opt, Ctx **out) {
  if (!systems || !out || nsys < 1) {
    set_error("cm3d_nb_create: null argument or no systems");
    return CM3D_NB_ERR_ARG;
  }
  cm3d_nb_options o;
  cm3d_nb_default_options(&o);
  if (opt) o = *opt;
  if (nsys > 1 && o.mode != CM3D_NB_MIXED) {
    set_error("cm3d_nb_create_batch: batches run in the mixed engine only (the plain FP64 engine is one system "
              "per context)");
    return CM3D_NB_ERR_ARG;
  }
  long long ntot = 0;
  for (int sy = 0; sy < nsys; sy++) {
    const cm3d_nb_system *s = systems + sy;
    if (s->natoms <= 0) {
      set_error("cm3d_nb_create: system %d: natoms = %d", sy, s->natoms);
      return CM3D_NB_ERR_ARG;
    }
    if (s->iperd != 3) {
      set_error("cm3d_nb_create: system %d: only iperd 3 (three-dimensional periodicity) is supported, got %d", sy,
                s->iperd);
      return CM3D_NB_ERR_ARG;
    }
    if (s->ntable < 5) {
      set_error("cm3d_nb_create: system %d: ntable = %d is too small", sy, s->ntable);
      return CM3D_NB_ERR_ARG;
    }
    // NVE, or NVT with Nose-Hoover chains (the same chain length in every
    // system of a batch); barostats (NPT) are not supported
    const bool nvt = s->iensemble == 1 && s->ntherm > 0 && s->nchain > 0 && s->ithm && s->mnh && s->gkt &&
                     s->nhc_eta && s->nhc_veta;
    if (!(s->iensemble == 0 && s->ntherm == 0) && !nvt) {
      set_error("cm3d_nb_create: system %d: ensemble %d with %d thermostats is not supported: the engine "
                "integrates NVE or NVT with Nose-Hoover chains, without barostats",
                sy, s->iensemble, s->ntherm);
      return CM3D_NB_ERR_ARG;
    }
    if (s->iensemble != systems[0].iensemble || (nvt && s->nchain != systems[0].nchain)) {
      set_error("cm3d_nb_create_batch: system %d: every system of a batch needs the same ensemble and chain length",
                sy);
      return CM3D_NB_ERR_ARG;
    }
    const cm3d_nb_system *s0 = systems;
    if (s->ntable != s0->ntable || s->dt != s0->dt || s->nres_lrf != s0->nres_lrf ||
        s->nres_intra != s0->nres_intra || s->nres_tors != s0->nres_tors) {
      set_error("cm3d_nb_create_batch: system %d differs from system 0 in ntable, dt or the RESPA levels; a batch "
                "steps all its systems together",
                sy);
      return CM3D_NB_ERR_ARG;
    }
    ntot += s->natoms;
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    set_error("cm3d_nb_create: no CUDA device (%s)", e != cudaSuccess ? cudaGetErrorString(e) : "count 0");
    return CM3D_NB_ERR_NODEV;
  }
  if (o.mode == CM3D_NB_MIXED && ntot > MAX_ATOMS_MIXED) {
    set_error("cm3d_nb_create: the mixed engine holds at most %d atoms per context", MAX_ATOMS_MIXED);
    return CM3D_NB_ERR_ARG;
  }
  Ctx *c = new Ctx();
  *out = c;
  c->dev = o.device;
  CK(cudaSetDevice(c->dev));
  CK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->dev));
  {
    int optin = 0;
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->dev));
    c->smem_optin = (size_t)optin;
    // CM3D_NB_PAIR_KERNEL=list keeps single systems on the list-gather pair
    // kernel (the one batches and small boxes use), for comparisons
    const char *pk = getenv("CM3D_NB_PAIR_KERNEL");
    if (pk && strcmp(pk, "list") == 0) c->win_ok = 0, c->win_env_off = 1;
  }
  CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
  c->mode = o.mode;
  c->need_short = o.need_short;
  c->tpa = o.tpa;
  c->use_graph = o.use_graph;
  c->cell_scale = o.cell_scale >= 1.0 ? o.cell_scale : 1.0;
  c->nsys = nsys;
  c->h_sp.assign(nsys, SysP());
  c->hs.assign(nsys, SysH());
  const cm3d_nb_system *s0 = systems;
  const int n = (int)ntot;
  c->n = n;
  c->ntable = s0->ntable;
  c->iperd = 3;
  c->nres_lrf = s0->nres_lrf > 0 ? s0->nres_lrf : 1;
  c->nres_intra = s0->nres_intra > 0 ? s0->nres_intra : 1;
  c->nres_tors = s0->nres_tors > 0 ? s0->nres_tors : 1;
  c->dt = s0->dt;
  const int nt = s0->ntable;
  // concatenated host arrays
  const size_t n3 = 3 * (size_t)n;
  std::vector<double> pos(n3), vel(n3), mass(n), q(n);
  std::vector<int> itype(n), sys_of(n), map, ich, eoff(n + 1, 0), eidx, coff(n + 1, 0), cidx;
  std::vector<double> vtab, dvtab, swt, icut, coultab, dcoultab, switchse;
  int a0 = 0, inter0 = 0, ncoul = 0;
  for (int sy = 0; sy < nsys; sy++) {
    const cm3d_nb_system *s = systems + sy;
    SysP &P = c->h_sp[sy];
    SysH &H = c->hs[sy];
    const int ns = s->natoms;
    P.a0 = a0;
    P.n = ns;
    H.n = ns;
    H.ndof = s->ndof > 0 ? s->ndof : 1;
    H.ntypes = s->ntypes;
    H.ninter = s->ninter;
    H.vlrc = s->vlrc;
    H.wlrc = s->wlrc;
    H.scale14 = s->n14 > 0 ? s->scale_onefour : 1.0;
    H.scale14e = s->n14 > 0 ? s->scale_onefour_e : 1.0;
    H.iperd = s->iperd;
    memcpy(H.hmat, s->hmat, sizeof H.hmat);
    box_params(P, H);
    P.kappa = s->kappa;
    P.kappa2 = s->kappa * s->kappa;
    P.falp2 = s->falp2;
    H.ewald_self = s->ewald_self;
    H.ewald_bkg = s->ewald_bkg;
    P.skin2q = .25 * s->skin_ter * s->skin_ter;
    // atoms
    for (int i = 0; i < ns; i++) {
      const int g = a0 + i;
      pos[g] = s->px[i];
      pos[n + g] = s->py[i];
      pos[2 * (size_t)n + g] = s->pz[i];
      vel[g] = s->vx ? s->vx[i] : 0.;
      vel[n + g] = s->vy ? s->vy[i] : 0.;
      vel[2 * (size_t)n + g] = s->vz ? s->vz[i] : 0.;
      mass[g] = s->amass[i];
      q[g] = s->qch[i];
      itype[g] = s->itype[i];
      sys_of[g] = sy;
      // charged atoms (set_charges, elec_ngbr.c:115-121)
      if (s->qch[i] != 0.) {
        ich.push_back(g);
        H.ncharge++;
      }
    }
    if (H.ncharge > 0 && (!s->coultab || !s->dcoultab)) {
      set_error("cm3d_nb_create: system %d: charged atoms but no coultab/dcoultab", sy);
      return CM3D_NB_ERR_ARG;
    }
    // exclusion lists (CSR over global atom indices)
    P.excl = P.cexcl = 0;
    for (int i = 0; i < ns; i++) {
      const int e0 = s->excl_off ? s->excl_off[i] : 0, e1 = s->excl_off ? s->excl_off[i + 1] : 0;
      for (int k = e0; k < e1; k++) eidx.push_back(a0 + s->excl_idx[k]);
      eoff[a0 + i + 1] = (int)eidx.size();
      const int c0 = s->cexcl_off ? s->cexcl_off[i] : 0, c1 = s->cexcl_off ? s->cexcl_off[i + 1] : 0;
      for (int k = c0; k < c1; k++) cidx.push_back(a0 + s->cexcl_idx[k]);
      coff[a0 + i + 1] = (int)cidx.size();
      if (e1 > e0) P.excl = 1;
      if (c1 > c0) P.cexcl = 1;
    }
    // interactions: global indices inter0 + local, type map per system
    P.ntypes = s->ntypes;
    P.map0 = (int)map.size();
    P.inter0 = inter0;
    P.ninter = s->ninter;
    for (int k = 0; k < s->ntypes * s->ntypes; k++) map.push_back(s->map[k] >= 0 ? inter0 + s->map[k] : -1);
    double r2 = 0;
    for (int in = 0; in < s->ninter; in++) {
      icut.push_back(s->rmaxs_cut2[in]);
      icut.push_back(s->rmins_cut2[in]);
      icut.push_back(s->rmaxl_cut2[in]);
      icut.push_back(s->rminl_cut2[in]);
      icut.push_back(s->rmaxs_skin2[in]);
      icut.push_back(s->rmaxl_skin2[in]);
      icut.push_back(s->dx2tab[in]);
      icut.push_back(s->vtab[(size_t)in * nt + nt - 4]);
      r2 = std::max(r2, s->rmaxl_skin2[in]);
      for (int k = 0; k < nt; k++) {
        vtab.push_back(s->vtab[(size_t)in * nt + k]);
        dvtab.push_back(s->dvtab[(size_t)in * nt + k]);
        swt.push_back(s->switchs ? s->switchs[(size_t)in * nt + k] : 0.0);
      }
    }
    inter0 += s->ninter;
    // charges: this system's erfc table and radii
    if (H.ncharge > 0) {
      P.coul = ncoul++;
      for (int k = 0; k < nt; k++) {
        coultab.push_back(s->coultab[k]);
        dcoultab.push_back(s->dcoultab[k]);
        switchse.push_back(s->switchse ? s->switchse[k] : 0.0);
      }
      P.rmaxl_skin2_e = s->rmaxl_skin2_e;
      P.rmaxs_skin2_e = s->rmaxs_skin2_e;
      H.rmaxl_coul2 = s->rmaxl_coul2;
      H.dx2coul = s->dx2coul;
      H.rmins_coul2 = s->rmins_coul2;
      P.rc2_el = (float)s->rmaxl_coul2;
      P.dx2c = (float)s->dx2coul;
      P.offc = (float)(s->rmins_coul2 * s->dx2coul);
      P.tablast_e = (float)s->coultab[nt - 4];
      r2 = std::max(r2, s->rmaxl_skin2_e);
      H.ktot = s->ktot;
      H.ka.assign(s->ka, s->ka + s->ktot);
      H.kb.assign(s->kb, s->kb + s->ktot);
      H.kc.assign(s->kc, s->kc + s->ktot);
    } else {
      P.coul = -1;
      P.rmaxl_skin2_e = P.rmaxs_skin2_e = -1.0;
    }
    H.rlist = sqrt(r2);
    H.skin = s->skin_ter;
    box_widths(P, H);
    a0 += ns;
  }
  c->ncoul = ncoul;
  c->ncharge = (int)ich.size();
  c->ninter = inter0;
  // the scalar fields describe system 0 (the plain engine and the single-system
  // paths read them)
  {
    const cm3d_nb_system *s = s0;
    const SysH &H = c->hs[0];
    c->ntypes = s->ntypes;
    c->ndof = H.ndof;
    c->vlrc = s->vlrc;
    c->wlrc = s->wlrc;
    c->skin = s->skin_ter;
    c->rheal = s->rheal;
    memcpy(c->hmat, H.hmat, sizeof c->hmat);
    memcpy(c->hmati, H.hmati, sizeof c->hmati);
    c->kappa = s->kappa;
    c->kappa2 = s->kappa * s->kappa;
    c->falp2 = s->falp2;
    c->ewald_self = s->ewald_self;
    c->ewald_bkg = s->ewald_bkg;
    c->dx2coul = s->dx2coul;
    c->rmins_coul2 = s->rmins_coul2;
    c->rmaxs_coul2 = s->rmaxs_coul2;
    c->rminl_coul2 = s->rminl_coul2;
    c->rmaxl_coul2 = s->rmaxl_coul2;
    c->rmaxs_skin2_e = s->rmaxs_skin2_e;
    c->rmaxl_skin2_e = s->rmaxl_skin2_e;
    c->necorr = s->necorr;
    c->nbonds = s->nbonds;
    c->nbends = s->nbends;
    c->tablast_e = H.ncharge > 0 ? s->coultab[nt - 4] : 0.0;
    c->rlist_max = H.rlist;
    for (int in = 0; in < s->ninter; in++) c->rc_lj_max = std::max(c->rc_lj_max, sqrt(s->rmaxl_cut2[in]));
  }
  // device arrays
  int rc;
  if ((rc = upload(&c->pos, pos.data(), n3))) return rc;
  if ((rc = upload(&c->vel, vel.data(), n3))) return rc;
  if ((rc = upload<double>(&c->fxl, nullptr, n3))) return rc;
  if ((rc = upload<double>(&c->fxs, nullptr, n3))) return rc;
  if ((rc = upload<double>(&c->fxa, nullptr, n3))) return rc;
  if ((rc = upload<double>(&c->fxr, nullptr, n3))) return rc;
  if ((rc = upload<double>(&c->dxn, pos.data(), n3))) return rc;
  if ((rc = upload(&c->mass, mass.data(), n))) return rc;
  if ((rc = upload(&c->q, q.data(), n))) return rc;
  if ((rc = upload(&c->itype, itype.data(), n))) return rc;
  if ((rc = upload(&c->sys_of, sys_of.data(), n))) return rc;
  if ((rc = upload(&c->map, map.data(), map.size()))) return rc;
  if ((rc = upload(&c->vtab, vtab.data(), vtab.size()))) return rc;
  if ((rc = upload(&c->dvtab, dvtab.data(), dvtab.size()))) return rc;
  if ((rc = upload(&c->switchs, swt.data(), swt.size()))) return rc;
  if ((rc = upload(&c->icut, icut.data(), icut.size()))) return rc;
  if ((rc = upload(&c->coultab, coultab.data(), coultab.size()))) return rc;
  if ((rc = upload(&c->dcoultab, dcoultab.data(), dcoultab.size()))) return rc;
  if ((rc = upload(&c->switchse, switchse.data(), switchse.size()))) return rc;
  if ((rc = upload(&c->excl_off, eoff.data(), eoff.size()))) return rc;
  if ((rc = upload(&c->excl_idx, eidx.data(), eidx.size()))) return rc;
  if ((rc = upload(&c->cexcl_off, coff.data(), coff.size()))) return rc;
  if ((rc = upload(&c->cexcl_idx, cidx.data(), cidx.size()))) return rc;
  if ((rc = upload(&c->icharge, ich.data(), ich.size()))) return rc;
  // accumulators: per system ACC_COUNT sums + device copies of hmati and hmat
  std::vector<double> acc0((size_t)nsys * ACC_STRIDE, 0.0);
  for (int sy = 0; sy < nsys; sy++)
    for (int k = 0; k < 9; k++) {
      acc0[(size_t)sy * ACC_STRIDE + ACC_COUNT + k] = c->hs[sy].hmati[k];
      acc0[(size_t)sy * ACC_STRIDE + ACC_COUNT + 9 + k] = c->hs[sy].hmat[k];
    }
  if ((rc = upload(&c->acc, acc0.data(), acc0.size()))) return rc;
  if ((rc = upload<long long>(&c->stat, nullptr, ST_COUNT))) return rc;
  if ((rc = upload<int>(&c->istate, nullptr, IS_COUNT))) return rc;
  if ((rc = upload<int>(&c->sreb, nullptr, (size_t)nsys))) return rc;
  if ((rc = upload<int>(&c->slast, nullptr, (size_t)nsys))) return rc;
  if ((rc = upload<long long>(&c->sstat, nullptr, (size_t)nsys * SS_COUNT))) return rc;
  CK(cudaMallocHost(&c->h_acc, sizeof(double) * (size_t)nsys * ACC_STRIDE));
  CK(cudaMallocHost(&c->h_stat, sizeof(long long) * ST_COUNT));
  CK(cudaMallocHost(&c->h_istate, sizeof(int) * IS_COUNT));
  CK(cudaMallocHost(&c->h_sstat, sizeof(long long) * (size_t)nsys * SS_COUNT));
  memset(c->h_istate, 0, sizeof(int) * IS_COUNT);
  if ((rc = list_setup(c))) return rc;
  if ((rc = pair_setup(c))) return rc;
  if ((rc = cw_setup(c))) return rc;
  if ((rc = kspace_setup(c))) return rc;
  if ((rc = step_setup(c, systems, nsys))) return rc;
  if ((rc = upload(&c->sp, c->h_sp.data(), c->h_sp.size()))) return rc;
  CK(cudaDeviceSynchronize());
  return CM3D_NB_OK;
}

// FMA throughput probe: 8 independent dependency chains per thread
template <typename T>
__global__ void k_fma_peak(T *out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = (T)(threadIdx.x + k);
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
#pragma unroll
      for (int k = 0; k < 8; k++) x[k] = x[k] * a + b;
    }
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += x[k];
  if (s == (T)-12345.0) out[0] = s;   // keeps the chains alive
}

template <typename T>
static double fma_peak(int blocks) {
  T *out = nullptr;
  if (cudaMalloc(&out, sizeof(T)) != cudaSuccess) return 0;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int threads = 256, iters = 4096;
  double best = 0;
  for (int rep = 0; rep < 6; rep++) {
    cudaEventRecord(a);
    k_fma_peak<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-7);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    if (rep > 0 && ms > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  return best;
}

__global__ void k_scale_rmass(int n, double *__restrict__ f, const double *__restrict__ mass) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double r = 1. / mass[i];
  f[i] *= r;
  f[n + i] *= r;
  f[2 * n + i] *= r;
}

static double *block_of(Ctx *c, int which) {
  return which == CM3D_NB_FXL   ? c->fxl
         : which == CM3D_NB_FXS ? c->fxs
         : which == CM3D_NB_FXA ? c->fxa
         : which == CM3D_NB_FXR ? c->fxr
                                : nullptr;
}

static int pull_acc(Ctx *c) {
  CK(cudaMemcpyAsync(c->h_acc, c->acc, sizeof(double) * (size_t)c->nsys * ACC_STRIDE, cudaMemcpyDeviceToHost,
                     c->st));
  CK(cudaStreamSynchronize(c->st));
  return CM3D_NB_OK;
}

static void sym9(const double *a, int base, double t[9]) {
  t[0] = a[base + 0];
  t[1] = a[base + 1];
  t[2] = a[base + 2];
  t[4] = a[base + 4];
  t[5] = a[base + 5];
  t[8] = a[base + 8];
  t[3] = t[1];
  t[6] = t[2];
  t[7] = t[5];
}

static double deth(const double *h) {
  return (h[0] * (h[4] * h[8] - h[5] * h[7]) + h[1] * (h[5] * h[6] - h[3] * h[8]) +
          h[2] * (h[3] * h[7] - h[4] * h[6]));
}

}  // namespace cm3d

using namespace cm3d;

extern "C" {

struct cm3d_nb_ctx {
  Ctx c;
};

int cm3d_nb_version(void) { return 10000; }

const char *cm3d_nb_last_error(void) { return g_err; }

int cm3d_nb_device_count(int *count) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (count) *count = e == cudaSuccess ? n : 0;
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
  return CM3D_NB_OK;
}

void cm3d_nb_default_options(cm3d_nb_options *opt) {
  opt->device = 0;
  opt->mode = CM3D_NB_MIXED;
  opt->need_short = 0;
  opt->tpa = 0;
  opt->use_graph = 1;
  opt->cell_scale = 1.0;
}

int cm3d_nb_create(const cm3d_nb_system *sys, const cm3d_nb_options *opt, cm3d_nb_ctx **out) {
  return cm3d_nb_create_batch(sys, 1, opt, out);
}

int cm3d_nb_create_batch(const cm3d_nb_system *systems, int nsys, const cm3d_nb_options *opt, cm3d_nb_ctx **out) {
  DevLock lock(device_mutex());
  Ctx *c = nullptr;
  int rc = create(systems, nsys, opt, &c);
  if (rc) {
    destroy(c);
    if (out) *out = nullptr;
    return rc;
  }
  *out = reinterpret_cast<cm3d_nb_ctx *>(c);
  return CM3D_NB_OK;
}

void cm3d_nb_destroy(cm3d_nb_ctx *ctx) {
  DevLock lock(device_mutex());
  destroy(reinterpret_cast<Ctx *>(ctx));
}

// every entry point first finishes asynchronously launched steps
#define CTX                                         \
  Ctx *c = reinterpret_cast<Ctx *>(ctx);            \
  if (!c) {                                         \
    set_error("null context");                      \
    return CM3D_NB_ERR_ARG;                         \
  }                                                 \
  do {                                              \
    cudaError_t _e = cudaSetDevice(c->dev);         \
    if (_e != cudaSuccess) return cuda_fail(_e, "cudaSetDevice"); \
    if (c->pending) {                               \
      int _rc = finish_steps(c);                    \
      if (_rc) return _rc;                          \
    }                                               \
  } while (0)

static int put3(Ctx *c, double *dst, const double *x, const double *y, const double *z) {
  const size_t n = c->n;
  CK(cudaMemcpyAsync(dst, x, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dst + n, y, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dst + 2 * n, z, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CM3D_NB_OK;
}

static int get3(Ctx *c, const double *src, double *x, double *y, double *z) {
  const size_t n = c->n;
  CK(cudaMemcpyAsync(x, src, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(y, src + n, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(z, src + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CM3D_NB_OK;
}

int cm3d_nb_set_positions(cm3d_nb_ctx *ctx, const double *px, const double *py, const double *pz) {
  CTX;
  return put3(c, c->pos, px, py, pz);
}
// A new box for a one-system context (a barostat's step): every parameter
// derived from H -- H^-1, the volume, the small-box test, the cell grid's
// neighbour shifts and the device copies the kernels read -- follows it; the
// grid keeps its cell counts, which stays valid while every cell is at least
// a list radius wide.
int cm3d_nb_set_box(cm3d_nb_ctx *ctx, const double hmat[9]) {
  CTX;
  DevLock lock(device_mutex());
  if (c->nsys != 1) {
    set_error("set_box: a batch of %d systems (one system only)", c->nsys);
    return CM3D_NB_ERR_ARG;
  }
  SysH H = c->hs[0];
  SysP P = c->h_sp[0];
  memcpy(H.hmat, hmat, sizeof H.hmat);
  box_params(P, H);
  if (!(P.rvol > 0.0) || !isfinite(P.rvol)) {
    set_error("set_box: a singular or left-handed box matrix");
    return CM3D_NB_ERR_ARG;
  }
  if (H.iperd == 3)
    for (int d = 0; d < 3; d++)
      if (box_width(H, d) / P.nc[d] < H.rlist) {
        set_error("set_box: the box shrank below the cell grid (%d cells of width %g < list radius %g along "
                  "direction %d); create a new context for this box",
                  P.nc[d], box_width(H, d) / P.nc[d], H.rlist, d);
        return CM3D_NB_ERR_STATE;
      }
  box_widths(P, H);
  cell_shifts(P, H);
  c->hs[0] = H;
  c->h_sp[0] = P;
  memcpy(c->hmat, H.hmat, sizeof c->hmat);
  memcpy(c->hmati, H.hmati, sizeof c->hmati);
  CK(cudaStreamSynchronize(c->st));
  CK(cudaMemcpy(c->sp, c->h_sp.data(), sizeof(SysP), cudaMemcpyHostToDevice));
  if (c->shift) {
    CK(cudaMemcpy(c->shift, P.shift, sizeof(float4) * 27, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->shift + 27, P.shift_lo, sizeof(float4) * 27, cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(c->acc + ACC_COUNT, H.hmati, sizeof(double) * 9, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->acc + ACC_COUNT + 9, H.hmat, sizeof(double) * 9, cudaMemcpyHostToDevice));
  // a captured step holds the old box in its launch parameters
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  return refresh_corners(c);
}

int cm3d_nb_get_positions(cm3d_nb_ctx *ctx, double *px, double *py, double *pz) {
  CTX;
  return get3(c, c->pos, px, py, pz);
}
int cm3d_nb_set_velocities(cm3d_nb_ctx *ctx, const double *vx, const double *vy, const double *vz) {
  CTX;
  return put3(c, c->vel, vx, vy, vz);
}
int cm3d_nb_get_velocities(cm3d_nb_ctx *ctx, double *vx, double *vy, double *vz) {
  CTX;
  return get3(c, c->vel, vx, vy, vz);
}
int cm3d_nb_get_forces(cm3d_nb_ctx *ctx, int which, double *fx, double *fy, double *fz) {
  CTX;
  double *b = block_of(c, which);
  if (!b) {
    set_error("get_forces: unknown block %d", which);
    return CM3D_NB_ERR_ARG;
  }
  return get3(c, b, fx, fy, fz);
}
int cm3d_nb_set_forces(cm3d_nb_ctx *ctx, int which, const double *fx, const double *fy, const double *fz) {
  CTX;
  double *b = block_of(c, which);
  if (!b) {
    set_error("set_forces: unknown block %d", which);
    return CM3D_NB_ERR_ARG;
  }
  return put3(c, b, fx, fy, fz);
}

int cm3d_nb_get_ngbr(cm3d_nb_ctx *ctx) {
  CTX;
  return build_lists(c, false, true);
}

int cm3d_nb_nrefsh(cm3d_nb_ctx *ctx, int istep, int *rebuilt) {
  CTX;
  int rc;
  if (rebuilt) *rebuilt = 0;
  if (!c->lists_built) {
    set_error("nrefsh() before get_ngbr()");
    return CM3D_NB_ERR_STATE;
  }
  c->h_istate[IS_ISTEP] = istep;
  CK(cudaMemcpyAsync(c->istate + IS_ISTEP, c->h_istate + IS_ISTEP, sizeof(int), cudaMemcpyHostToDevice, c->st));
  if ((rc = check_displacement(c))) return rc;
  if ((rc = reset_positions(c))) return rc;
  CK(cudaMemcpyAsync(c->h_istate, c->istate, sizeof(int) * IS_COUNT, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (c->h_istate[IS_REBUILD]) {
    if ((rc = build_lists(c, false, false))) return rc;
    if (rebuilt) *rebuilt = 1;
  }
  return CM3D_NB_OK;
}

int cm3d_nb_force(cm3d_nb_ctx *ctx, int iflg) {
  CTX;
  return run_force(c, iflg);
}

// zero accumulator slots [first, first + count) of every system
static int zero_slots(Ctx *c, int first, int count) {
  CK(cudaMemset2DAsync(c->acc + first, sizeof(double) * ACC_STRIDE, 0, sizeof(double) * count, (size_t)c->nsys,
                       c->st));
  return CM3D_NB_OK;
}

int cm3d_nb_force_ter(cm3d_nb_ctx *ctx, int iflg) {
  CTX;
  if (!c->lists_built) {
    set_error("force_ter() before get_ngbr()");
    return CM3D_NB_ERR_STATE;
  }
  if (iflg != 0 && iflg != 1) {
    set_error("force_ter(): level must be 0 or 1");
    return CM3D_NB_ERR_ARG;
  }
  int rc;
  if (iflg == 1 && (rc = zero_slots(c, ACC_SPOTL, 12))) return rc;   // zero_potl md_fnopol.c:38
  return pair_forces(c, iflg, 1);
}

int cm3d_nb_force_ter_e(cm3d_nb_ctx *ctx, int iflg) {
  CTX;
  if (!c->lists_built) {
    set_error("force_ter_e() before get_ngbr()");
    return CM3D_NB_ERR_STATE;
  }
  if (iflg != 0 && iflg != 1) {
    set_error("force_ter_e(): level must be 0 or 1");
    return CM3D_NB_ERR_ARG;
  }
  int rc;
  if (iflg == 1 && (rc = zero_slots(c, ACC_SPOTE, 12))) return rc;   // zero_pote finter_e.c:34
  return pair_forces(c, iflg, 2);
}

int cm3d_nb_fk_ewald(cm3d_nb_ctx *ctx) {
  CTX;
  int rc;
  if ((rc = zero_slots(c, ACC_VK, 11))) return rc;
  return kspace_forces(c);
}

int cm3d_nb_ecorr(cm3d_nb_ctx *ctx) {
  CTX;
  int rc;
  if ((rc = zero_slots(c, ACC_POT_ECORR, 11))) return rc;
  return plain_ecorr(c, c->ecorr_pairs);
}

int cm3d_nb_zero_forces(cm3d_nb_ctx *ctx, int which) {
  CTX;
  double *b = block_of(c, which);
  if (!b) {
    set_error("zero_forces: unknown block %d", which);
    return CM3D_NB_ERR_ARG;
  }
  CK(cudaMemsetAsync(b, 0, sizeof(double) * 3 * (size_t)c->n, c->st));
  return CM3D_NB_OK;
}

int cm3d_nb_rmass(cm3d_nb_ctx *ctx, int which) {
  CTX;
  double *b = block_of(c, which);
  if (!b) {
    set_error("rmass: unknown block %d", which);
    return CM3D_NB_ERR_ARG;
  }
  k_scale_rmass<<<grid_for(c->n, 256), 256, 0, c->st>>>(c->n, b, c->mass);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

int cm3d_nb_getsvirter(cm3d_nb_ctx *ctx, double *vhinter, double *vinter, double *winter, double wintert[9]) {
  CTX;
  int rc;
  if ((rc = pull_acc(c))) return rc;
  double t[9];
  sym9(c->h_acc, ACC_SPRSLT, t);
  *vhinter += c->h_acc[ACC_SPOTHL];
  *vinter += c->h_acc[ACC_SPOTL];
  *winter += c->h_acc[ACC_SPRSL];
  for (int k = 0; k < 9; k++) wintert[k] += t[k];
  return CM3D_NB_OK;
}

int cm3d_nb_getsvirter_e(cm3d_nb_ctx *ctx, double *velec, double *welec, double welectensor[9]) {
  CTX;
  int rc;
  if ((rc = pull_acc(c))) return rc;
  double t[9];
  sym9(c->h_acc, ACC_SPRSET, t);
  *velec += c->h_acc[ACC_SPOTE];
  *welec += c->h_acc[ACC_SPRSE];
  for (int k = 0; k < 9; k++) welectensor[k] += t[k];
  return CM3D_NB_OK;
}

// fk_ewald's totals (md_ewald.c:336-348) plus ecorr, as getvewald adds
// them, for system `sy` (pulled accumulators)
static void ewald_totals(Ctx *c, int sy, double *pot, double *prs, double tens[9]) {
  const SysH &H = c->hs[sy];
  const double *a = c->h_acc + (size_t)sy * ACC_STRIDE;
  double six = H.ncharge > 0 ? H.ewald_bkg / deth(H.hmat) : 0.0;
  double vk = a[ACC_VK], vp = a[ACC_VP];
  double vk_ewald = 0, vp_ewald = 0, vpt[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (H.iperd == 3) {
    vk_ewald = vk + six + (H.ncharge > 0 ? H.ewald_self : 0.0);
    vp_ewald = vp + 3. * (vk + six);
    for (int k = 0; k < 9; k++) vpt[k] = a[ACC_VPT + k];
    vpt[0] += vk + six;
    vpt[4] += vk + six;
    vpt[8] += vk + six;
  }
  double ct[9];
  sym9(a, ACC_PRS_ECORRT, ct);
  *pot = vk_ewald + a[ACC_POT_ECORR];
  *prs = vp_ewald + a[ACC_PRS_ECORR];
  for (int k = 0; k < 9; k++) tens[k] = vpt[k] + ct[k];
}

int cm3d_nb_getvewald(cm3d_nb_ctx *ctx, double *pot_ewald, double *prs_ewald, double prs_ewald_tensor[9]) {
  CTX;
  int rc;
  if ((rc = pull_acc(c))) return rc;
  double p, w, t[9];
  ewald_totals(c, 0, &p, &w, t);
  *pot_ewald += p;
  *prs_ewald += w;
  for (int k = 0; k < 9; k++) prs_ewald_tensor[k] += t[k];
  return CM3D_NB_OK;
}

int cm3d_nb_step_init(cm3d_nb_ctx *ctx) {
  CTX;
  int rc;
  c->h_istate[IS_ISTEP] = 0;
  c->h_istate[IS_ISTEPLAST] = 0;
  CK(cudaMemcpyAsync(c->istate, c->h_istate, sizeof(int) * 2, cudaMemcpyHostToDevice, c->st));
  if ((rc = build_lists(c, false, true))) return rc;
  if ((rc = run_force(c, 1))) return rc;
  if ((rc = run_force(c, 2))) return rc;
  if ((rc = run_force(c, 3))) return rc;
  c->forces_valid = true;
  return CM3D_NB_OK;
}

int cm3d_nb_step(cm3d_nb_ctx *ctx, int istep0, int nsteps) {
  CTX;
  return run_step(c, istep0, nsteps);
}

int cm3d_nb_set_host_outputs(cm3d_nb_ctx *ctx, double *pos_out, double *vel_out) {
  CTX;
  DevLock lock(device_mutex());
  if (c->pending) {
    set_error("set_host_outputs: asynchronous steps are in flight (cm3d_nb_step_wait first)");
    return CM3D_NB_ERR_STATE;
  }
  for (double *p : {pos_out, vel_out}) {
    if (!p) continue;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess || a.type != cudaMemoryTypeHost) {
      cudaGetLastError();
      set_error("set_host_outputs: %p is not page-locked host memory (cudaMallocHost / cudaHostRegister)", (void *)p);
      return CM3D_NB_ERR_ARG;
    }
  }
  if ((pos_out || vel_out) && !c->st3) {
    CK(cudaStreamCreateWithFlags(&c->st3, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->ev_f3, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_j3, cudaEventDisableTiming));
  }
  c->ho_pos = pos_out;
  c->ho_vel = vel_out;
  if (c->graph) {                           // captured with the old outputs
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  return CM3D_NB_OK;
}

int cm3d_nb_step_host(cm3d_nb_ctx *ctx, int istep0, const double *pos_in, const double *vel_in) {
  CTX;
  if (c->pending) {
    set_error("step_host: asynchronous steps are in flight (cm3d_nb_step_wait first)");
    return CM3D_NB_ERR_STATE;
  }
  const size_t b = sizeof(double) * 3 * (size_t)c->n;
  if (pos_in) CK(cudaMemcpyAsync(c->pos, pos_in, b, cudaMemcpyHostToDevice, c->st));
  if (vel_in) CK(cudaMemcpyAsync(c->vel, vel_in, b, cudaMemcpyHostToDevice, c->st));
  return run_step(c, istep0, 1);
}

int cm3d_nb_step_async(cm3d_nb_ctx *ctx, int istep0, int nsteps) {
  CTX;
  return launch_steps(c, istep0, nsteps);
}

int cm3d_nb_step_query(cm3d_nb_ctx *ctx, int *done) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || !done) {
    set_error("step_query: null argument");
    return CM3D_NB_ERR_ARG;
  }
  cudaError_t e = cudaSetDevice(c->dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  return query_steps(c, done);
}

int cm3d_nb_step_wait(cm3d_nb_ctx *ctx) {
  CTX;   // finishes the pending steps
  return CM3D_NB_OK;
}

// getvireal(...,1)+geteng() of system `sy` from the pulled accumulators
static void energies_of(Ctx *c, int sy, cm3d_nb_energies *e) {
  const SysH &H = c->hs[sy];
  const double *a = c->h_acc + (size_t)sy * ACC_STRIDE;
  memset(e, 0, sizeof *e);
  e->vinter = a[ACC_SPOTL];
  e->vhinter = a[ACC_SPOTHL];
  e->winter = a[ACC_SPRSL];
  sym9(a, ACC_SPRSLT, e->wintertensor);
  e->velec = a[ACC_SPOTE];
  e->welec = a[ACC_SPRSE];
  sym9(a, ACC_SPRSET, e->welectensor);
  ewald_totals(c, sy, &e->vewald, &e->wewald, e->wewaldtensor);
  e->vbond = a[ACC_VBOND];
  e->wbond = a[ACC_WBOND];
  e->vbend = a[ACC_VBEND];
  e->wbend = a[ACC_WBEND];
  double vol = deth(H.hmat), rvol = 1. / vol;
  e->US = e->vhinter + e->velec + e->vewald;
  e->U = e->vinter + e->velec + e->vewald;
  e->W = e->winter + e->welec + e->wewald;
  for (int k = 0; k < 9; k++) e->Wtensor[k] = e->wintertensor[k] + e->welectensor[k] + e->wewaldtensor[k];
  e->W -= 3 * H.wlrc * rvol;
  e->Wtensor[0] -= H.wlrc * rvol;
  e->Wtensor[4] -= H.wlrc * rvol;
  e->Wtensor[8] -= H.wlrc * rvol;
  sym9(a, ACC_P2MT, e->p2m_tensor);
  double p2m = e->p2m_tensor[0] + e->p2m_tensor[4] + e->p2m_tensor[8];
  // torsions (virial = the tensor's trace, md_ftors.c:532), 1-4 pairs scaled
  // as getvonfo scales its sums (md_fonefour.c:303-312); the 1-4 Coulomb
  // virial equals its energy term by term
  e->vtors = a[ACC_VTORS];
  e->wtors = a[ACC_WTORST + 0] + a[ACC_WTORST + 4] + a[ACC_WTORST + 8];
  e->vonfo = a[ACC_VONFO] * H.scale14;
  e->wonfo = a[ACC_WONFO] * H.scale14;
  e->vonfo_e = a[ACC_VONFO_E] * H.scale14e;
  e->wonfo_e = a[ACC_VONFO_E] * H.scale14e;
  e->UI = e->vbond + e->vbend + e->vtors + e->vonfo + e->vonfo_e;
  e->WI = e->wbond + e->wbend + e->wtors + e->wonfo + e->wonfo_e;
  for (int k = 0; k < 9; k++)
    e->WItensor[k] = a[ACC_WBONDT + k] + a[ACC_WBENDT + k] + a[ACC_WTORST + k] + a[ACC_WONFOT + k] * H.scale14 +
                     a[ACC_WONFOET + k] * H.scale14e + a[ACC_WBONDXT + k];
  e->poth = e->US + H.vlrc / vol;
  e->poter = e->U + H.vlrc / vol;
  e->potra = e->UI;
  e->prsi = (p2m + e->W + e->WI) / (3 * vol);
  for (int k = 0; k < 9; k++) e->prs_tensor[k] = (e->p2m_tensor[k] + e->Wtensor[k] + e->WItensor[k]) / vol;
  e->zke = .5 * p2m;
  e->tiout = p2m / (double)H.ndof;
}

int cm3d_nb_get_energies(cm3d_nb_ctx *ctx, cm3d_nb_energies *e) {
  return cm3d_nb_get_system_energies(ctx, 0, e);
}

int cm3d_nb_get_system_energies(cm3d_nb_ctx *ctx, int sys, cm3d_nb_energies *e) {
  CTX;
  int rc;
  if (sys < 0 || sys >= c->nsys) {
    set_error("get_system_energies: system %d of %d", sys, c->nsys);
    return CM3D_NB_ERR_ARG;
  }
  if ((rc = pull_acc(c))) return rc;
  energies_of(c, sys, e);
  return CM3D_NB_OK;
}

int cm3d_nb_get_all_energies(cm3d_nb_ctx *ctx, cm3d_nb_energies *e) {
  CTX;
  int rc;
  if ((rc = pull_acc(c))) return rc;
  for (int s = 0; s < c->nsys; s++) energies_of(c, s, e + s);
  return CM3D_NB_OK;
}

int cm3d_nb_num_systems(cm3d_nb_ctx *ctx, int *nsys) {
  CTX;
  *nsys = c->nsys;
  return CM3D_NB_OK;
}

int cm3d_nb_system_atoms(cm3d_nb_ctx *ctx, int sys, int *first, int *natoms) {
  CTX;
  if (sys < 0 || sys >= c->nsys) {
    set_error("system_atoms: system %d of %d", sys, c->nsys);
    return CM3D_NB_ERR_ARG;
  }
  *first = c->h_sp[sys].a0;
  *natoms = c->h_sp[sys].n;
  return CM3D_NB_OK;
}

int cm3d_nb_system_counts(cm3d_nb_ctx *ctx, long long *rebuilds, long long *resets) {
  CTX;
  CK(cudaMemcpyAsync(c->h_sstat, c->sstat, sizeof(long long) * (size_t)c->nsys * SS_COUNT, cudaMemcpyDeviceToHost,
                     c->st));
  CK(cudaStreamSynchronize(c->st));
  for (int s = 0; s < c->nsys; s++) {
    if (rebuilds) rebuilds[s] = c->h_sstat[(size_t)s * SS_COUNT + SS_REBUILDS];
    if (resets) resets[s] = c->h_sstat[(size_t)s * SS_COUNT + SS_RESETS];
  }
  return CM3D_NB_OK;
}

int cm3d_nb_get_nhc(cm3d_nb_ctx *ctx, int sys, double *eta, double *veta, int *ntherm, int *nchain) {
  CTX;
  if (sys < 0 || sys >= c->nsys) {
    set_error("get_nhc: system %d of %d", sys, c->nsys);
    return CM3D_NB_ERR_ARG;
  }
  const int nt = c->ntherm > 0 ? c->therm0[(size_t)sys + 1] - c->therm0[(size_t)sys] : 0;
  if (ntherm) *ntherm = nt;
  if (nchain) *nchain = c->ntherm > 0 ? c->nchain : 0;
  if (nt == 0) return CM3D_NB_OK;
  const size_t tc = (size_t)c->ntherm * c->nchain, o = (size_t)c->therm0[(size_t)sys] * c->nchain,
               k = (size_t)nt * c->nchain;
  CK(cudaStreamSynchronize(c->st));
  if (eta) CK(cudaMemcpy(eta, c->nhc + 2 * tc + o, sizeof(double) * k, cudaMemcpyDeviceToHost));
  if (veta) CK(cudaMemcpy(veta, c->nhc + 3 * tc + o, sizeof(double) * k, cudaMemcpyDeviceToHost));
  return CM3D_NB_OK;
}

// The mixed engine's rebuilds write only its full list.  CM3D's half lists
// are produced on request by rebuilding from the positions of the last
// rebuild (dxn): the same cells and the same pairs, without touching the
// live state or the snapshot.
static int ensure_half_lists(Ctx *c) {
  if (c->mode != CM3D_NB_MIXED || !c->lists_built) return CM3D_NB_OK;
  std::swap(c->pos, c->dxn);
  c->want_half = true;
  c->no_snapshot = true;
  int rc = build_lists(c, false, true);
  std::swap(c->pos, c->dxn);
  c->want_half = false;
  c->no_snapshot = false;
  return rc;
}

int cm3d_nb_list_count(cm3d_nb_ctx *ctx, int which, long long *npairs) {
  CTX;
  if (which < 0 || which > 3) {
    set_error("list_count: unknown list %d", which);
    return CM3D_NB_ERR_ARG;
  }
  int rc = ensure_half_lists(c);
  if (rc) return rc;
  *npairs = c->lists_built ? c->hcount[which] : 0;
  if (c->lists_built && c->use_graph && c->mode == CM3D_NB_PLAIN_FP64) {
    // device-gated rebuilds may have changed the counts since the host looked
    CK(cudaMemcpyAsync(c->h_ltot, c->ltot, sizeof(long long) * LT_COUNT, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int k = 0; k < LT_COUNT; k++) c->hcount[k] = c->h_ltot[k];
    *npairs = c->hcount[which];
  }
  return CM3D_NB_OK;
}

int cm3d_nb_get_list(cm3d_nb_ctx *ctx, int which, int *ip, int *jp, long long capacity, long long *npairs) {
  CTX;
  long long np = 0;
  int rc = cm3d_nb_list_count(ctx, which, &np);
  if (rc) return rc;
  if (npairs) *npairs = np;
  if (np > capacity) {
    set_error("get_list: %lld pairs do not fit in %lld", np, capacity);
    return CM3D_NB_ERR_ARG;
  }
  if (np == 0) return CM3D_NB_OK;
  std::vector<int2> h((size_t)np);
  CK(cudaMemcpyAsync(h.data(), c->lst[which], sizeof(int2) * (size_t)np, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  for (long long k = 0; k < np; k++) {
    ip[k] = h[k].x;
    jp[k] = h[k].y;
  }
  return CM3D_NB_OK;
}

int cm3d_nb_get_status(cm3d_nb_ctx *ctx, cm3d_nb_status_t *st) {
  CTX;
  CK(cudaMemcpyAsync(c->h_stat, c->stat, sizeof(long long) * ST_COUNT, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(c->h_istate, c->istate, sizeof(int) * IS_COUNT, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  st->table_underflow = c->h_stat[ST_UNDERFLOW];
  st->rebuilds = c->h_stat[ST_REBUILDS];
  st->resets = c->h_stat[ST_RESETS];
  st->overflows = c->overflows_host;
  st->nonfinite = (int)c->h_stat[ST_NONFINITE];
  st->last_istep = c->h_istate[IS_ISTEP];
  st->stage_timeouts = (int)c->h_stat[ST_STAGE_TIMEOUT];
  return CM3D_NB_OK;
}

int cm3d_nb_synchronize(cm3d_nb_ctx *ctx) {
  CTX;
  CK(cudaStreamSynchronize(c->st));
  return CM3D_NB_OK;
}

void *cm3d_nb_stream(cm3d_nb_ctx *ctx) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  return c ? (void *)c->st : nullptr;
}

int cm3d_nb_enable_timing(cm3d_nb_ctx *ctx, int enable) {
  CTX;
  collect_timing(c);
  c->timing.on = (enable & 1) != 0;
  c->timing.steps = (enable & 2) != 0;
  for (int k = 0; k < NTCLS; k++) {
    c->timing.ms[k] = 0;
    c->timing.launches[k] = 0;
  }
  return CM3D_NB_OK;
}

int cm3d_nb_kernel_time(cm3d_nb_ctx *ctx, int cls, double *ms, long long *launches) {
  CTX;
  if (cls < 0 || cls >= NTCLS) {
    set_error("kernel_time: unknown class %d", cls);
    return CM3D_NB_ERR_ARG;
  }
  collect_timing(c);
  if (ms) *ms = c->timing.ms[cls];
  if (launches) *launches = c->timing.launches[cls];
  return CM3D_NB_OK;
}

long long cm3d_nb_launch_count(cm3d_nb_ctx *ctx) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  return c ? c->launches : 0;
}

int cm3d_nb_pair_kernel(cm3d_nb_ctx *ctx, int *kernel, int *tpa) {
  CTX;
  if (kernel) *kernel = c->pair_used;
  if (tpa) *tpa = c->tpa;
  return CM3D_NB_OK;
}

int cm3d_nb_grid(cm3d_nb_ctx *ctx, int sys, int nc[3], int *nsplit, int *block_threads) {
  CTX;
  if (sys < 0 || sys >= c->nsys) {
    set_error("grid: system %d of %d", sys, c->nsys);
    return CM3D_NB_ERR_ARG;
  }
  if (nc)
    for (int d = 0; d < 3; d++) nc[d] = c->h_sp[sys].nc[d];
  if (nsplit) *nsplit = c->cw_ok ? c->cw_nsplit : 1;
  if (block_threads)
    *block_threads = !c->cw_ok ? 0 : (c->cw_batch && c->cw_row == CM3D_CS_LPA ? CM3D_CS_THREADS : c->cw_nt);
  return CM3D_NB_OK;
}

int cm3d_nb_autotune(cm3d_nb_ctx *ctx, int reps, int *tpa_chosen, double ms_per_launch[4]) {
  CTX;
  DevLock lock(device_mutex());
  int rc;
  if (c->mode != CM3D_NB_MIXED) {
    set_error("autotune: the plain FP64 engine has nothing to tune");
    return CM3D_NB_ERR_ARG;
  }
  if (!c->lists_built) {
    set_error("autotune before get_ngbr()/step_init(): it times the live lists");
    return CM3D_NB_ERR_STATE;
  }
  if (reps < 1) reps = 5;
  const int cand[4] = {4, 8, 16, 32};
  double best = 1e300;
  int best_tpa = c->tpa, best_win = 0, best_cw = 0, best_split = c->cw_nsplit, best_nt = c->cw_nt;
  int best_row = c->cw_row;
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  const bool timing = c->timing.on;
  c->timing.on = false;
  if (ms_per_launch)
    for (int k = 0; k < 4; k++) ms_per_launch[k] = 1e300;
  // kind 0: the gather kernel; 1: the staged kernel that applies (a single
  // system's 27-cell windows, or a batch's whole systems); 2: the compact
  // window list (nb_cwin.cu), 32 lanes per atom; 3: a batch's compact list
  // with 8 lanes per atom (k_pair_cs) -- the context runs whichever is
  // fastest on its live lists
  for (int kind = 0; kind <= 3; kind++) {
    if (kind == 1 && c->win_env_off) continue;
    if (kind >= 2 && !c->cw_ok) continue;
    if (kind == 3 && (!c->cw_batch || c->cw_cap8 == 0)) continue;
    c->win_ok = kind == 1;
    if (kind >= 2) {
      const int row = kind == 3 ? CM3D_CS_LPA : CM3D_CW_ROW;
      if (!c->cw_use) {
        // the compact lists are kept only while the compact path is in use:
        // convert every system's master list first
        c->cw_use = 1;
        if (c->cw_batch) {
          c->cw_row = row;
          c->cw_cap = row == CM3D_CS_LPA ? c->cw_cap8 : c->cw_cap32;
        }
        if ((rc = cw_convert(c, false, true))) return rc;
      } else if ((rc = cw_set_row(c, row))) {
        return rc;
      }
      if (!c->cw_ok) continue;                       // a window did not fit
      if (c->cw_batch && c->cw_row != row) continue;  // nor the 8-lane kernel's window
    }
    c->cw_use = kind >= 2;
    // the compact kernel runs a warp per atom; its tile is the number of
    // parts each cell's atoms are split into (work items per cell, each
    // staging the cell's window): 1, 2, 4, 8.  In a batch the lanes per
    // atom are those of the gather kernel that runs the other systems, and
    // the items are whole cells.
    for (int k = 0; k < 4; k++)
      for (int sp = 1; sp <= (kind == 2 && !c->cw_batch ? CW_MAX_SPLIT : 1); sp *= 2)
      for (int nt = 512; nt <= (kind == 2 ? 640 : 512); nt += 128) {
        if (kind == 2 && cand[k] != 32 && !c->cw_batch) continue;
        c->tpa = cand[k];
        if (kind == 2) {
          cw_set_split(c, sp);
          c->cw_nt = nt;
        }
        if ((rc = pair_forces(c, 1, 3))) return rc;   // warm-up (first launch sets attributes)
        CK(cudaEventRecord(a, c->st));
        for (int r = 0; r < reps; r++)
          if ((rc = pair_forces(c, 1, 3))) return rc;
        CK(cudaEventRecord(b, c->st));
        CK(cudaEventSynchronize(b));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, a, b));
        const double per = ms / reps;
        if (ms_per_launch && per < ms_per_launch[k]) ms_per_launch[k] = per;
        if (per < best) {
          best = per;
          best_tpa = cand[k];
          best_win = kind == 1;
          best_cw = kind >= 2;
          if (kind >= 2) {
            best_split = sp;
            best_nt = nt;
            best_row = kind == 3 ? CM3D_CS_LPA : CM3D_CW_ROW;
          }
        }
      }
  }
  c->timing.on = timing;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  c->tpa = best_tpa;
  c->win_ok = best_win;
  c->cw_use = best_cw;
  if (c->cw_ok) {
    cw_set_split(c, best_split);
    c->cw_nt = best_nt;
    if (best_cw && (rc = cw_set_row(c, best_row))) return rc;
  }
  if (tpa_chosen) *tpa_chosen = best_tpa;
  // a captured step holds the old launch configuration; the timing launches
  // added to the force blocks and accumulators: recompute force(1)
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  if ((rc = run_force(c, 1))) return rc;
  CK(cudaStreamSynchronize(c->st));
  return CM3D_NB_OK;
}

int cm3d_nb_measure_peaks(int device, double *fp32_tflops, double *fp64_tflops) {
  CK(cudaSetDevice(device));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  if (fp32_tflops) *fp32_tflops = fma_peak<float>(sms * 16);
  if (fp64_tflops) *fp64_tflops = fma_peak<double>(sms * 16);
  CKL(nullptr);
  return CM3D_NB_OK;
}

// ------------------------------------------------- host set-up restatements
// func_lj  energy/inter/md_funcvdw.c:40-46
static void func_lj(double x, double *f, double *df, double eps, double sig) {
  *f = 4. * eps * (pow(sig / x, 12.) - pow(sig / x, 6.));
  *df = 4. * eps * (6. * pow(sig, 6.) * pow(x, -7.) - 12. * pow(sig, 12.) * pow(x, -13.));
  *df /= x;
}

// func_kerf  md_funcvdw.c:219-227 ; func_coul md_funcvdw.c:243-249
static void func_kerf(double x, double *f, double *df, double alpha) {
  *f = erfc(alpha * x) / x;
  *df = -erfc(alpha * x) / (x * x) - 2. * alpha * exp(-alpha * alpha * x * x) / (sqrt(M_PI) * x);
  *df /= x;
}
static void func_coul(double x, double *f, double *df) {
  *f = 1. / x;
  *df = -1. / (x * x);
  *df /= x;
}

int cm3d_nb_lj_table(double eps, double sig, double rmin, double rmax, double rres, double rheal, double skin,
                     int ntable, int shift, double *vtab, double *dvtab, double *switchs, double *dx2tab) {
  if (ntable < 5 || rmax <= rmin || !vtab || !dvtab || !switchs || !dx2tab) {
    set_error("lj_table: bad arguments (ntable %d, rmin %g, rmax %g)", ntable, rmin, rmax);
    return CM3D_NB_ERR_ARG;
  }
  // get_ter_parm md_getparm.c:222-254
  double rmins, rminl, rres_dist = rres;
  if (rres < rmax) {
    rmins = rmin;
    rminl = rres - rheal;
  } else {
    rmins = rmin;
    rminl = rmax + 2. * skin;
    rres_dist = rmax + 2. * rheal;
  }
  *dx2tab = ((double)ntable - 3.) / (rmax * rmax - rmin * rmin);
  if (rminl - skin < rmin) {
    set_error("lj_table: RESPA distance, healing length, skin and minimum distance are inconsistent");
    return CM3D_NB_ERR_ARG;
  }
  double rch = (rres_dist - rheal);
  double rhl = rheal == 0. ? 1. : 1. / rheal;
  for (int i = 0; i < ntable; i++) {
    double xt = i / (*dx2tab) + rmins * rmins, f, df;
    if (xt < 0) {
      set_error("lj_table: negative table abscissa");
      return CM3D_NB_ERR_ARG;
    }
    func_lj(sqrt(xt), &f, &df, eps, sig);
    vtab[i] = f * 1.0;     // scaleeps = 1 (md_setsimdef.c:63)
    dvtab[i] = df * 1.0;
    if (xt <= rch * rch) switchs[i] = 1.0;
    if (xt > rch * rch && xt < rres_dist * rres_dist) {
      double br = (sqrt(xt) - rch) * rhl, sm = (1. + br * br * (2. * br - 3.));
      switchs[i] = sm;
    }
    if (xt >= rres_dist * rres_dist) switchs[i] = 0.0;
  }
  if (shift) {
    double vs = vtab[ntable - 3];   // md_searchbase.c:181-188
    for (int i = 0; i < ntable; i++) vtab[i] -= vs;
  }
  return CM3D_NB_OK;
}

int cm3d_nb_coul_table(double alpha, double rcute_min, double rcute_resp, double rcute_max, double rheal,
                       double skin, int ntable, int iperd, int shift, double *coultab, double *dcoultab,
                       double *switchse, double *dx2coul) {
  (void)skin;
  if (ntable < 5 || rcute_max <= rcute_min || !coultab || !dcoultab || !switchse || !dx2coul) {
    set_error("coul_table: bad arguments");
    return CM3D_NB_ERR_ARG;
  }
  // set_charges elec_ngbr.c:51-103
  double rmins2 = rcute_min * rcute_min, rmaxs2 = rcute_resp * rcute_resp;
  double rminl2 = ((rcute_resp - rheal) * (rcute_resp - rheal)), rmaxl2 = rcute_max * rcute_max;
  *dx2coul = (((double)ntable - 3.) / (rmaxl2 - rmins2));
  for (int i = 0; i < ntable; i++) {
    double xt = i / *dx2coul + rmins2, f, df;
    if (xt < 0) {
      set_error("coul_table: negative table abscissa");
      return CM3D_NB_ERR_ARG;
    }
    if (iperd == 3) func_kerf(sqrt(xt), &f, &df, alpha);
    else func_coul(sqrt(xt), &f, &df);
    coultab[i] = f;
    dcoultab[i] = df;
    if (xt <= rminl2) switchse[i] = 1.;
    if (xt > rminl2 && xt < rmaxs2) {
      double br = (sqrt(xt) - sqrt(rminl2)) / rheal, sm = (1. + br * br * (2. * br - 3.));
      switchse[i] = sm;
    }
    if (xt >= rmaxs2) switchse[i] = 0.;
  }
  if (shift) {
    double vs = coultab[ntable - 3];
    for (int i = 0; i < ntable; i++) coultab[i] -= vs;
  }
  return CM3D_NB_OK;
}

int cm3d_nb_ewald_kvectors(int kmax, int *ka, int *kb, int *kc, int *kup, int *ktot) {
  // ewald_setup md_ewald.c:93-114: half space ka >= 0, spherical cutoff
  int n = 0, ksqmax = kmax * kmax;
  for (int i = 0; i <= kmax; i++)
    for (int j = (i == 0) ? 0 : -kmax; j <= kmax; j++) {
      int first = 1;
      for (int k = (i == 0 && j == 0) ? 1 : -kmax; k <= kmax; k++) {
        if (i * i + j * j + k * k <= ksqmax) {
          if (ka) {
            ka[n] = i;
            kb[n] = j;
            kc[n] = k;
            if (kup) kup[n] = first;
          }
          first = 0;
          n++;
        }
      }
    }
  if (ka && kup) kup[n] = 0;
  *ktot = n;
  return CM3D_NB_OK;
}

}  // extern "C"
