/*
 * cm3d_nb_shim.c -- CM3D's step_init() and step() (integrate/md_step.c:32-159)
 * on the B200 nonbonded engine, as a drop-in for CM3D's own md_step.o.
 *
 * Linked into CM3D in place of md_step.o (that object defines exactly these
 * two functions), it lets CM3D's unmodified MD driver (md_mdcntr_new,
 * main/md_mdcntr.new.c:174-178: step, geteng, gettngbr every step) run the
 * whole RESPA step on the GPU:
 *
 *   step_init  builds the engine's system description from CM3D's own
 *              SIMPARMS / COORDS / INTER structs once, uploads it
 *              (cm3d_nb_create), runs CM3D's step_init sequence on the device
 *              (cm3d_nb_step_init: get_ngbr, force(1), force(2),
 *              force(3)), and fills
 *              CM3D's ENERGIES the way getvireal(..., 1) does
 *              (energy/control/md_fcntr.c:136-257), then calls CM3D's own
 *              geteng and gettngbr as md_step.c:53-55 does;
 *   step       advances one outer step on the device (cm3d_nb_step with
 *              SIMPARMS.istep), copies positions and velocities back into
 *              COORDS (CM3D's writers and geteng read them) and refills
 *              ENERGIES.
 *
 * NVT (Nose-Hoover chains, intnhc_new in md_step.c:117): CM3D's chain state
 * (COORDS.eta / veta / mnh / gkt, SIMPARMS.ntherm / nchain, ithm) goes to
 * the engine at step_init, and after every step the chains' eta and veta
 * come back into COORDS, where CM3D's thermostat energy (getengn) and its
 * restart writer read them.
 *
 * What the engine does not compute -- barostats (npt_*), external fields,
 * dipoles, non-periodic boxes, the phased cosine torsion form -- stops the
 * run through md_error with the reason, as CM3D reports unsupported input;
 * nothing falls back to a CPU path.
 *
 * Environment: CM3D_NB_MODE=plain selects the plain FP64 engine (default:
 * mixed), CM3D_NB_DEVICE the CUDA device (default 0).
 *
 * Compiled with -DCM3D_NB_ROUTE_B the same file is the routine-level
 * binding instead: CM3D keeps its own step() and host integrator
 * (md_step.c, thermostat included), and only the nonbonded routines go to
 * the engine --
 *
 *   get_ngbr   (energy/control/ngbr_list.c:297, with get_ngbr_e) the
 *              engine's four lists from the current positions;
 *   nrefsh     (energy/control/md_finter.c:43) the engine's skin test and
 *              RESETPOS pull-back (cm3d_nb_nrefsh), positions read back;
 *   force      (energy/control/md_fcntr.c:44) every level on the engine,
 *              positions in and the level's force block out per call;
 *   getvireal  (energy/control/md_fcntr.c:136) ENERGIES from the engine's
 *              accumulators, as for route A.
 *
 * With a barostat (npt_i, npt_f: intbar in md_step.c moves COORDS.hmat) each
 * call hands the engine the current box first (cm3d_nb_set_box).
 *
 * CM3D's objects that define these four (md_fcntr.o, md_finter.o,
 * ngbr_list.o) are linked as copies in which the four symbols are weak, so
 * that the definitions here take their place (cm3d_b200/shim/Makefile).
 */
#include "md.h"

#include "cm3d_nb.h"

static cm3d_nb_ctx *g_ctx = NULL;
static int *g_map = NULL, *g_eoff = NULL, *g_eidx = NULL, *g_coff = NULL, *g_cidx = NULL;
static double *g_v14 = NULL, *g_dv14 = NULL;
static double *g_nhc = NULL;   /* NVT: mnh | gkt | eta | veta, ntherm * nchain each (row-major) */

static void nb_fail(const char *what)
{
  char line[1400];
  snprintf(line, sizeof line, "GPU nonbonded engine: %s: %s", what, cm3d_nb_last_error());
  md_error(line);
}

static void nb_check(int rc, const char *what)
{
  if (rc != CM3D_NB_OK) nb_fail(what);
}

static void unsupported(const char *what)
{
  char line[400];
  snprintf(line, sizeof line, "GPU nonbonded engine: %s is not supported", what);
  md_error(line);
}

/* the features the engine computes (see the file header) */
static void check_supported(SIMPARMS *simparms, COORDS *coords)
{
  if (simparms->iperd != 3) unsupported("a non-periodic or partially periodic box (iperd != 3)");
#ifndef CM3D_NB_ROUTE_B
  /* route B: CM3D's own step integrates the chains and the barostat on the
     host, and the engine follows the box (cm3d_nb_set_box) */
  if (simparms->iensemble != 0 && simparms->iensemble != 1)
    unsupported("a barostat (an ensemble other than nve or nvt)");
  if (simparms->ivol) unsupported("a variable cell (ivol)");
#endif
  if (simparms->iextern) unsupported("an external field");
  if (simparms->ipolar) unsupported("polarizable dipoles");
  (void)coords;
}

/* CSR copy of CM3D's per-atom exclusion lists (INTER.nexclude/exclude,
   COUL.nexclude/exclude) */
static void csr(int n, const int *cnt, int **lists, int **off, int **idx)
{
  int i, k, tot = 0;
  for (i = 0; i < n; i++) tot += cnt ? cnt[i] : 0;
  *off = (int *)malloc(sizeof(int) * (n + 1));
  *idx = (int *)malloc(sizeof(int) * (tot > 0 ? tot : 1));
  (*off)[0] = 0;
  for (i = 0; i < n; i++) {
    int c = cnt ? cnt[i] : 0;
    for (k = 0; k < c; k++) (*idx)[(*off)[i] + k] = lists[i][k];
    (*off)[i + 1] = (*off)[i] + c;
  }
}

static void create_engine(SIMPARMS *simparms, COORDS *coords, INTER *inter)
{
  cm3d_nb_system s;
  cm3d_nb_options opt;
  const char *mode = getenv("CM3D_NB_MODE"), *dev = getenv("CM3D_NB_DEVICE");
  int nt = simparms->ntypes, a, b;

  memset(&s, 0, sizeof s);
  s.natoms = simparms->natoms;
  s.iperd = simparms->iperd;
  s.nres_lrf = simparms->ninter;
  s.nres_intra = simparms->ninnra;
  s.nres_tors = simparms->ninrra;
  s.ndof = simparms->ndof;
  s.dt = simparms->dt;
  s.vlrc = simparms->vlrc;
  s.wlrc = simparms->wlrc;
  memcpy(s.hmat, coords->hmat, sizeof s.hmat);
  s.px = coords->px; s.py = coords->py; s.pz = coords->pz;
  s.vx = coords->vx; s.vy = coords->vy; s.vz = coords->vz;
  s.amass = coords->amass;
  s.qch = coords->qch;
  s.ntypes = nt;
  s.itype = inter->itype;
  g_map = (int *)malloc(sizeof(int) * (size_t)(nt * nt > 0 ? nt * nt : 1));
  for (a = 0; a < nt; a++)
    for (b = 0; b < nt; b++) g_map[a * nt + b] = inter->map[a][b];
  s.map = g_map;
  s.ninter = inter->ntype;
  s.ntable = inter->ntable;
  s.vtab = inter->ntype ? inter->vtab[0] : NULL;
  s.dvtab = inter->ntype ? inter->dvtab[0] : NULL;
  s.switchs = inter->ntype ? inter->switchs[0] : NULL;
  s.rmaxs_cut2 = inter->rmaxs_cut2;
  s.rmins_cut2 = inter->rmins_cut2;
  s.rmaxl_cut2 = inter->rmaxl_cut2;
  s.rminl_cut2 = inter->rminl_cut2;
  s.rmaxs_skin2 = inter->rmaxs_skin2;
  s.rmaxl_skin2 = inter->rmaxl_skin2;
  s.dx2tab = inter->dx2tab;
  s.skin_ter = inter->skin_ter;
  s.rheal = inter->rheal;
  if (coords->coul.ncharge > 0) {
    s.coultab = inter->coultab;
    s.dcoultab = inter->dcoultab;
    s.switchse = inter->switchse;
  }
  s.dx2coul = inter->dx2coul;
  s.rmins_coul2 = inter->rmins_coul2;
  s.rmaxs_coul2 = inter->rmaxs_coul2;
  s.rminl_coul2 = inter->rminl_coul2;
  s.rmaxl_coul2 = inter->rmaxl_coul2;
  s.rmaxs_skin2_e = inter->rmaxs_skin2_e;
  s.rmaxl_skin2_e = inter->rmaxl_skin2_e;
  csr(s.natoms, inter->nexclude, inter->exclude, &g_eoff, &g_eidx);
  csr(s.natoms, coords->coul.nexclude, coords->coul.exclude, &g_coff, &g_cidx);
  s.excl_off = g_eoff; s.excl_idx = g_eidx;
  s.cexcl_off = g_coff; s.cexcl_idx = g_cidx;
  s.ktot = coords->coul.ktot;
  s.ka = coords->coul.ka; s.kb = coords->coul.kb; s.kc = coords->coul.kc;
  s.kappa = coords->coul.kappa;
  s.falp2 = coords->coul.falp2;
  s.ewald_self = coords->coul.ewald_self;
  s.ewald_bkg = coords->coul.ewald_bkg;
  s.necorr = coords->coul.necorr;
  s.iecorr = coords->coul.iecorr;
  s.jecorr = coords->coul.jecorr;
  s.nbonds = coords->bonds.nbonds;
  s.nbond_types = coords->bonds.itypes;
  s.ibond = coords->bonds.ibond; s.jbond = coords->bonds.jbond;
  s.idxbond = coords->bonds.idxbond; s.itypbond = coords->bonds.itypbond;
  s.eqbond = coords->bonds.eqbond; s.fkbond = coords->bonds.fkbond;
  s.nbends = coords->bends.nbends;
  s.nbend_types = coords->bends.itypes;
  s.ibend = coords->bends.ibend; s.jbend = coords->bends.jbend; s.kbend = coords->bends.kbend;
  s.idxbend = coords->bends.idxbend; s.itypbend = coords->bends.itypbend;
  s.eqbend = coords->bends.eqbend; s.fkbend = coords->bends.fkbend;
  /* torsions, 1-4 pairs, cross bonds (TORS / ONFO / BONDXS) */
  s.ntors = coords->tors.ntorss;
  if (s.ntors > 0) {
    int t, nh = 0, nv = 0;
    s.ntors_types = coords->tors.itypes;
    s.itors = coords->tors.itors; s.jtors = coords->tors.jtors;
    s.ktors = coords->tors.ktors; s.ltors = coords->tors.ltors;
    s.idxtors = coords->tors.idxtors;
    s.tors_ind_pot = coords->tors.ind_pot;
    s.tors_ind_pot_num = coords->tors.ind_pot_num;
    for (t = 0; t < coords->tors.itypes; t++) {
      int k = coords->tors.ind_pot_num[t] + 1;
      if (coords->tors.ind_pot[t] == 0 && k > nh) nh = k;
      if (coords->tors.ind_pot[t] == 1 && k > nv) nv = k;
    }
    s.ntors_harm = nh;
    s.eqtors = coords->tors.eqtors; s.fktors = coords->tors.fktors;
    s.ntors_series = nv;
    s.vphi = nv > 0 ? &coords->tors.vphi[0][0] : NULL;
  }
  s.n14 = coords->onfo.n14s;
  if (s.n14 > 0) {
    /* ONFO's tables are rows of a dmatrix: copy them into one block */
    int t, nt14 = coords->onfo.itypes, nk = coords->onfo.n14table;
    g_v14 = (double *)malloc(sizeof(double) * (size_t)nt14 * nk);
    g_dv14 = (double *)malloc(sizeof(double) * (size_t)nt14 * nk);
    for (t = 0; t < nt14; t++) {
      memcpy(g_v14 + (size_t)t * nk, coords->onfo.v14tab[t], sizeof(double) * nk);
      memcpy(g_dv14 + (size_t)t * nk, coords->onfo.dv14tab[t], sizeof(double) * nk);
    }
    s.n14_types = nt14;
    s.n14table = nk;
    s.i14 = coords->onfo.i14; s.j14 = coords->onfo.j14; s.i14dx = coords->onfo.i14dx;
    s.r14min2 = coords->onfo.r14min2; s.r14max2 = coords->onfo.r14max2;
    s.dx214tab = coords->onfo.dx214tab;
    s.v14tab = g_v14; s.dv14tab = g_dv14;
    s.scale_onefour = coords->onfo.scale_onefour;
    s.scale_onefour_e = coords->onfo.scale_onefour_e;
  }
  s.nbondx = coords->bondxs.nbondxs;
  if (s.nbondx > 0) {
    s.nbondx_types = coords->bondxs.itypes;
    s.ibondx = coords->bondxs.ibondx; s.jbondx = coords->bondxs.jbondx;
    s.kbondx = coords->bondxs.kbondx; s.idxbondx = coords->bondxs.idxbox;
    s.eq1bondx = coords->bondxs.eq1bondx; s.eq2bondx = coords->bondxs.eq2bondx;
    s.fkbondx = coords->bondxs.fkbondx;
  }
  s.nfreeze = simparms->nfreeze;
  s.ifreeze = coords->ifreeze;
#ifndef CM3D_NB_ROUTE_B
  if (simparms->iensemble == 1) {
    /* CM3D's chains are dmatrix rows [ntherm][nchain]: flat copies */
    int j, k, nt = simparms->ntherm, nc = simparms->nchain;
    size_t tc = (size_t)nt * nc;
    g_nhc = (double *)malloc(sizeof(double) * 4 * (tc > 0 ? tc : 1));
    for (j = 0; j < nt; j++)
      for (k = 0; k < nc; k++) {
        g_nhc[(size_t)j * nc + k] = coords->mnh[j][k];
        g_nhc[tc + (size_t)j * nc + k] = coords->gkt[j][k];
        g_nhc[2 * tc + (size_t)j * nc + k] = coords->eta[j][k];
        g_nhc[3 * tc + (size_t)j * nc + k] = coords->veta[j][k];
      }
    s.iensemble = 1;
    s.ntherm = nt;
    s.nchain = nc;
    s.ithm = coords->ithm;
    s.mnh = g_nhc;
    s.gkt = g_nhc + tc;
    s.nhc_eta = g_nhc + 2 * tc;
    s.nhc_veta = g_nhc + 3 * tc;
  }
#endif

  cm3d_nb_default_options(&opt);
  if (mode && strcmp(mode, "plain") == 0) opt.mode = CM3D_NB_PLAIN_FP64;
  if (dev) opt.device = atoi(dev);
  nb_check(cm3d_nb_create(&s, &opt, &g_ctx), "cm3d_nb_create");
}

/* ENERGIES as getvireal(..., 1) leaves them (md_fcntr.c:136-257): the engine
   supplies every nonbonded, Ewald and bonded term; the terms it does not
   compute are zero */
static void fill_energies(SIMPARMS *simparms, COORDS *coords, ENERGIES *energies)
{
  cm3d_nb_energies e;
  int i;
  nb_check(cm3d_nb_get_energies(g_ctx, &e), "cm3d_nb_get_energies");
  energies->vinter = e.vinter;
  energies->vhinter = e.vhinter;
  energies->velec = e.velec;
  energies->vewald = e.vewald;
  energies->vbond = e.vbond;
  energies->vbend = e.vbend;
  energies->vtors = e.vtors;
  energies->vonfo = e.vonfo;
  energies->vonfo_e = e.vonfo_e;
  energies->vbondx = 0.0;             /* getvbondx adds into vbond (md_fcntr.c:182) */
  energies->vextern = energies->vextern_e = 0.0;
  energies->winter = e.winter;
  energies->welec = e.welec;
  energies->wewald = e.wewald;
  energies->wbond = e.wbond;
  energies->wbend = e.wbend;
  energies->wtors = e.wtors;
  energies->wonfo = e.wonfo;
  energies->wonfo_e = e.wonfo_e;
  energies->wbondx = 0.0;
  energies->wextern = energies->wextern_e = 0.0;
  energies->US = e.US;
  energies->U = e.U;
  energies->W = e.W;
  energies->UI = e.UI;
  energies->WI = e.WI;
  for (i = 0; i < 9; i++) {
    energies->wintertensor[i] = e.wintertensor[i];
    energies->welectensor[i] = e.welectensor[i];
    energies->wewaldtensor[i] = e.wewaldtensor[i];
    energies->Wtensor[i] = e.Wtensor[i];
    /* the intramolecular virial tensor as one sum (CM3D reads only the sum) */
    energies->WItensor[i] = e.WItensor[i];
    energies->wbondtensor[i] = energies->WItensor[i];
    energies->wbendtensor[i] = energies->wtorstensor[i] = energies->wbondxtensor[i] = 0.0;
    energies->wonfotensor[i] = energies->wonfo_etensor[i] = 0.0;
  }
  (void)simparms;
  (void)coords;
}

static void pull_state(SIMPARMS *simparms, COORDS *coords)
{
  nb_check(cm3d_nb_get_positions(g_ctx, coords->px, coords->py, coords->pz), "cm3d_nb_get_positions");
  nb_check(cm3d_nb_get_velocities(g_ctx, coords->vx, coords->vy, coords->vz), "cm3d_nb_get_velocities");
  if (g_nhc) {
    /* the chains as the step left them (cm3d_nb_get_nhc) into COORDS */
    int j, k, nt = simparms->ntherm, nc = simparms->nchain;
    size_t tc = (size_t)nt * nc;
    nb_check(cm3d_nb_get_nhc(g_ctx, 0, g_nhc + 2 * tc, g_nhc + 3 * tc, NULL, NULL), "cm3d_nb_get_nhc");
    for (j = 0; j < nt; j++)
      for (k = 0; k < nc; k++) {
        coords->eta[j][k] = g_nhc[2 * tc + (size_t)j * nc + k];
        coords->veta[j][k] = g_nhc[3 * tc + (size_t)j * nc + k];
      }
  }
}

static void pull_forces(COORDS *coords)
{
  nb_check(cm3d_nb_get_forces(g_ctx, CM3D_NB_FXL, coords->fxl, coords->fyl, coords->fzl), "get_forces");
  nb_check(cm3d_nb_get_forces(g_ctx, CM3D_NB_FXS, coords->fxs, coords->fys, coords->fzs), "get_forces");
  nb_check(cm3d_nb_get_forces(g_ctx, CM3D_NB_FXA, coords->fxa, coords->fya, coords->fza), "get_forces");
  nb_check(cm3d_nb_get_forces(g_ctx, CM3D_NB_FXR, coords->fxr, coords->fyr, coords->fzr), "get_forces");
}

/* NGBR as get_ngbr leaves it (energy/control/ngbr_list.c:308): the pair
   counts of the current lists, and update = list builds so far - 1 (step_init
   sets -1 and its first build makes it 0), which writescreen turns into
   <ts/update> (output/md_writescreen.c:48-64) */
static void list_counts(NGBR *ngbr)
{
  long long c;
  cm3d_nb_status_t st;
  nb_check(cm3d_nb_get_status(g_ctx, &st), "get_status");
  ngbr->update = (int)(st.rebuilds - 1);
  nb_check(cm3d_nb_list_count(g_ctx, CM3D_NB_LIST_T, &c), "list_count"); ngbr->nprt = (int)c;
  nb_check(cm3d_nb_list_count(g_ctx, CM3D_NB_LIST_S, &c), "list_count"); ngbr->nprs = (int)c;
  nb_check(cm3d_nb_list_count(g_ctx, CM3D_NB_LIST_TE, &c), "list_count"); ngbr->nprte = (int)c;
  nb_check(cm3d_nb_list_count(g_ctx, CM3D_NB_LIST_SE, &c), "list_count"); ngbr->nprse = (int)c;
}

#ifndef CM3D_NB_ROUTE_B
void step_init(SIMPARMS *simparms, COORDS *coords, ENERGIES *energies, INTER *inter, NGBR *ngbr)
{
  check_supported(simparms, coords);
  if (simparms->rank == 0) md_stdout("Calculating initial forces (B200 nonbonded engine)");
  if (!g_ctx) {
    create_engine(simparms, coords, inter);
  } else {
    nb_check(cm3d_nb_set_positions(g_ctx, coords->px, coords->py, coords->pz), "set_positions");
    nb_check(cm3d_nb_set_velocities(g_ctx, coords->vx, coords->vy, coords->vz), "set_velocities");
  }
  nb_check(cm3d_nb_step_init(g_ctx), "step_init");
  pull_forces(coords);
  list_counts(ngbr);
  fill_energies(simparms, coords, energies);
  geteng(simparms, coords, energies);
  gettngbr(ngbr);
}

void step(SIMPARMS *simparms, COORDS *coords, ENERGIES *energies, INTER *inter, NGBR *ngbr)
{
  (void)inter;
  nb_check(cm3d_nb_step(g_ctx, simparms->istep, 1), "step");
  pull_state(simparms, coords);
  list_counts(ngbr);
  fill_energies(simparms, coords, energies);
  gettngbr(ngbr);
}
#else /* CM3D_NB_ROUTE_B */

static double g_box[9];

/* the current box (when a barostat moved it) and positions to the engine */
static void push_positions(COORDS *coords)
{
  if (memcmp(g_box, coords->hmat, sizeof g_box) != 0) {
    nb_check(cm3d_nb_set_box(g_ctx, coords->hmat), "set_box");
    memcpy(g_box, coords->hmat, sizeof g_box);
  }
  nb_check(cm3d_nb_set_positions(g_ctx, coords->px, coords->py, coords->pz), "set_positions");
}

/* get_ngbr (energy/control/ngbr_list.c:297): the first call -- from CM3D's
   step_init -- creates the engine from SIMPARMS / COORDS / INTER; every call
   builds the engine's lists from COORDS' positions and sets NGBR's pair
   counts and update (CM3D's own host lists are not built) */
void get_ngbr(SIMPARMS *simparms, COORDS *coords, INTER *inter, NGBR *ngbr)
{
  if (!g_ctx) {
    check_supported(simparms, coords);
    create_engine(simparms, coords, inter);
    memcpy(g_box, coords->hmat, sizeof g_box);
  } else {
    push_positions(coords);
  }
  nb_check(cm3d_nb_get_ngbr(g_ctx), "get_ngbr");
  list_counts(ngbr);
}

/* nrefsh (energy/control/md_finter.c:43): the skin test against the last
   build's positions, RESETPOS, and the rebuild, on the engine; a rebuild
   may have pulled positions back, so COORDS gets them again */
void nrefsh(SIMPARMS *simparms, COORDS *coords, INTER *inter, NGBR *ngbr)
{
  int rebuilt = 0;
  (void)inter;
  push_positions(coords);
  nb_check(cm3d_nb_nrefsh(g_ctx, simparms->istep, &rebuilt), "nrefsh");
  if (rebuilt) {
    nb_check(cm3d_nb_get_positions(g_ctx, coords->px, coords->py, coords->pz), "get_positions");
    list_counts(ngbr);
  }
}

/* force (energy/control/md_fcntr.c:44): the level on the engine, its force
   block(s) back as accelerations; frozen atoms' velocities go through the
   engine's freeze_atom too */
void force(SIMPARMS *simparms, COORDS *coords, INTER *inter, NGBR *ngbr, int iflg)
{
  (void)inter;
  (void)ngbr;
  push_positions(coords);
  if (simparms->nfreeze > 0)
    nb_check(cm3d_nb_set_velocities(g_ctx, coords->vx, coords->vy, coords->vz), "set_velocities");
  nb_check(cm3d_nb_force(g_ctx, iflg), "force");
  switch (iflg) {
    case 1:
      nb_check(cm3d_nb_get_forces(g_ctx, CM3D_NB_FXL, coords->fxl, coords->fyl, coords->fzl), "get_forces");
      /* fall through: level 1 also refills fxs */
    case 0:
      nb_check(cm3d_nb_get_forces(g_ctx, CM3D_NB_FXS, coords->fxs, coords->fys, coords->fzs), "get_forces");
      break;
    case 2:
      nb_check(cm3d_nb_get_forces(g_ctx, CM3D_NB_FXA, coords->fxa, coords->fya, coords->fza), "get_forces");
      break;
    case 3:
      nb_check(cm3d_nb_get_forces(g_ctx, CM3D_NB_FXR, coords->fxr, coords->fyr, coords->fzr), "get_forces");
      break;
    default:
      md_error("force: level out of range");
  }
  if (simparms->nfreeze > 0)
    nb_check(cm3d_nb_get_velocities(g_ctx, coords->vx, coords->vy, coords->vz), "get_velocities");
}

/* getvireal (energy/control/md_fcntr.c:136) for iflg 1, the only form
   CM3D's step and step_init use: the engine's accumulators of the last
   force(1) and its bonded terms */
void getvireal(SIMPARMS *simparms, COORDS *coords, ENERGIES *energies, INTER *inter, NGBR *ngbr, int iflg)
{
  (void)inter;
  (void)ngbr;
  if (iflg != 1) md_error("GPU nonbonded engine: getvireal is bound for iflg 1 only");
  fill_energies(simparms, coords, energies);
}
#endif /* CM3D_NB_ROUTE_B */
