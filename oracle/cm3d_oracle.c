/*
 * cm3d_oracle.c -- CPU restatement of CM3D's nonbonded force path.
 *
 * TEST INFRASTRUCTURE ONLY (see cm3d_oracle.h).  Every function restates the
 * CM3D routine named in its comment, keeping CM3D's operation order so that
 * the results match the reference bit for bit when compiled without FMA
 * contraction (-ffp-contract=off): pair lists in link-cell traversal order,
 * pair kernels over nlen-sized chunks with per-chunk energy partials, the
 * Ewald kc-recursion, and the same accumulation order of every sum.
 */
#include "cm3d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* include/md_macros.h:52 (LINUX build): round half away from zero through a
   truncating int conversion */
#define ANINT(A) ((int)((A) + ((A) >= 0 ? .5 : -.5)))
#define TPI (2. * M_PI)
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

struct orc {
  int n, ntypes, ninter, ntable, ncells, nocell_all, nlen, iperd;
  int nres_lrf, nres_intra, nres_tors, ndof;
  double dt, vlrc, wlrc, skin, rheal;
  double hmat[9], hmati[9];
  double *px, *py, *pz, *vx, *vy, *vz, *amass, *qch;
  int *itype, *map;
  double *vtab, *dvtab, *switchs;
  double *rmaxs_cut2, *rmins_cut2, *rmaxl_cut2, *rminl_cut2, *rmaxs_skin2,
      *rmaxl_skin2, *dx2tab;
  double *coultab, *dcoultab, *switchse;
  double dx2coul, rmins_coul2, rmaxs_coul2, rminl_coul2, rmaxl_coul2,
      rmaxs_skin2_e, rmaxl_skin2_e;
  int *excl_off, *excl_idx, *cexcl_off, *cexcl_idx;
  int ncharge, *icharge;
  int ktot, *ka, *kb, *kc, *kup;
  double kappa, kappa2, falp2, ewald_self, ewald_bkg;
  int necorr, *iecorr, *jecorr;
  int nbonds, *ibond, *jbond, *idxbond, *itypbond;
  double *eqbond, *fkbond;
  int nbends, *ibend, *jbend, *kbend, *idxbend, *itypbend;
  double *eqbend, *fkbend;
  /* forces (3n blocks: x | y | z), scratch, neighbour state */
  double *fxl, *fxs, *fxa, *scr, *rec, *dxn;
  long long nprt, nprs, nprte, nprse, cap_t, cap_s, cap_te, cap_se;
  int *inpt, *jnpt, *inps, *jnps, *inpte, *jnpte, *inpse, *jnpse;
  int npaircell, *icell, *jcell, npaircelle, *icelle, *jcelle;
  int *hlist, *lnk, cells_ready;
  int isteplast;
  long long rebuilds, resets, underflows;
  /* module statics of md_fnopol.c:33, finter_e.c:31, COUL accumulators */
  double spotl, spothl, sprsl, sprslt[9];
  double spote, spothe, sprse, sprset[9];
  double vk_ewald, vp_ewald, vp_ewald_tensor[9];
  double pot_ecorr, prs_ecorr, prs_ecorr_tensor[9];
  double vbond, wbond, wbondt[9], vbend, wbend, wbendt[9];
  /* TORS / ONFO / BONDXS (md_typedef.h:81-100) and the torsion-level forces */
  int ntors, *itors, *jtors, *ktors, *ltors, *idxtors, *tors_form, *tors_row;
  double *eqtors, *fktors, *vphi;
  int n14, n14table, *i14, *j14, *i14dx;
  double *r14min2, *r14max2, *dx214tab, *v14tab, *dv14tab, scale14, scale14e;
  int nbondx, *ibondx, *jbondx, *kbondx, *idxbondx;
  double *eq1bondx, *eq2bondx, *fkbondx;
  double *fxr;
  int nfreeze, *ifreeze;
  /* Nose-Hoover chains (SIMPARMS.ntherm / nchain, COORDS.ithm, mnh, gkt,
     eta, veta, feta, p2mt) */
  int ntherm, nchain, *ithm;
  double *mnh, *gkt, *eta, *veta, *feta, *p2mt;
  double vtors, wtors, wtorst[9], vonfo, vonfo_e, wonfo, wonfo_e, wonfot[9], wonfoet[9], wbondxt[9];
};

static void *dup(const void *p, size_t bytes)
{
  void *q = malloc(bytes > 0 ? bytes : 1);
  if (p && bytes) memcpy(q, p, bytes);
  else memset(q, 0, bytes > 0 ? bytes : 1);
  return q;
}

/* gethinv9  utils/md_mathlib.c:30-50 */
static double gethinv9(const double h[9], double hi[9])
{
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
  return 1. / rvol;
}

/* get_deth  utils/md_mathlib.c:53-60 */
static double get_deth(const double h[9])
{
  return (h[0] * (h[4] * h[8] - h[5] * h[7]) + h[1] * (h[5] * h[6] - h[3] * h[8]) +
          h[2] * (h[3] * h[7] - h[4] * h[6]));
}

/* period_new  integrate/md_period.new.c:39-52 (iperd 3) */
static void period(int n, double *dx, double *dy, double *dz, const double *h,
                   const double *hi)
{
  int j;
  for (j = 0; j < n; j++) {
    double sx = dx[j] * hi[0] + dy[j] * hi[1] + dz[j] * hi[2];
    double sy = dx[j] * hi[3] + dy[j] * hi[4] + dz[j] * hi[5];
    double sz = dx[j] * hi[6] + dy[j] * hi[7] + dz[j] * hi[8];
    sx -= ANINT(sx);
    sy -= ANINT(sy);
    sz -= ANINT(sz);
    dx[j] = sx * h[0] + sy * h[1] + sz * h[2];
    dy[j] = sx * h[3] + sy * h[4] + sz * h[5];
    dz[j] = sx * h[6] + sy * h[7] + sz * h[8];
  }
}

/* locate/exclij  utils/utils.c:125-172: is (i, j) in the sorted exclusion
   list stored at the lower index */
static int exclij(int i, int j, const int *off, const int *idx)
{
  int a = i < j ? i : j, b = i < j ? j : i;
  int lo = off[a], hi = off[a + 1];
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (idx[mid] == b) return 1;
    if (idx[mid] < b) lo = mid + 1;
    else hi = mid;
  }
  return 0;
}

orc *orc_create(const cm3d_nb_system *s, int ncells, int nocell_all, int nlen)
{
  orc *o = (orc *)calloc(1, sizeof(orc));
  int n = s->natoms, i, nt = s->ntable, ni = s->ninter;
  o->n = n;
  o->ntypes = s->ntypes;
  o->ninter = ni;
  o->ntable = nt;
  o->ncells = ncells;
  o->nocell_all = nocell_all;
  o->nlen = nlen;
  o->iperd = s->iperd;
  o->nres_lrf = s->nres_lrf;
  o->nres_intra = s->nres_intra;
  o->nres_tors = s->nres_tors;
  o->ndof = s->ndof;
  o->dt = s->dt;
  o->vlrc = s->vlrc;
  o->wlrc = s->wlrc;
  o->skin = s->skin_ter;
  o->rheal = s->rheal;
  memcpy(o->hmat, s->hmat, sizeof o->hmat);
  gethinv9(o->hmat, o->hmati);
  o->px = (double *)dup(s->px, n * 8.);
  o->py = (double *)dup(s->py, n * 8.);
  o->pz = (double *)dup(s->pz, n * 8.);
  o->vx = (double *)dup(s->vx, n * 8.);
  o->vy = (double *)dup(s->vy, n * 8.);
  o->vz = (double *)dup(s->vz, n * 8.);
  o->amass = (double *)dup(s->amass, n * 8.);
  o->qch = (double *)dup(s->qch, n * 8.);
  o->itype = (int *)dup(s->itype, n * 4.);
  o->map = (int *)dup(s->map, (size_t)s->ntypes * s->ntypes * 4);
  o->vtab = (double *)dup(s->vtab, (size_t)ni * nt * 8);
  o->dvtab = (double *)dup(s->dvtab, (size_t)ni * nt * 8);
  o->switchs = (double *)dup(s->switchs, (size_t)ni * nt * 8);
  o->rmaxs_cut2 = (double *)dup(s->rmaxs_cut2, ni * 8.);
  o->rmins_cut2 = (double *)dup(s->rmins_cut2, ni * 8.);
  o->rmaxl_cut2 = (double *)dup(s->rmaxl_cut2, ni * 8.);
  o->rminl_cut2 = (double *)dup(s->rminl_cut2, ni * 8.);
  o->rmaxs_skin2 = (double *)dup(s->rmaxs_skin2, ni * 8.);
  o->rmaxl_skin2 = (double *)dup(s->rmaxl_skin2, ni * 8.);
  o->dx2tab = (double *)dup(s->dx2tab, ni * 8.);
  o->coultab = (double *)dup(s->coultab, s->coultab ? nt * 8. : 0);
  o->dcoultab = (double *)dup(s->dcoultab, s->dcoultab ? nt * 8. : 0);
  o->switchse = (double *)dup(s->switchse, s->switchse ? nt * 8. : 0);
  o->dx2coul = s->dx2coul;
  o->rmins_coul2 = s->rmins_coul2;
  o->rmaxs_coul2 = s->rmaxs_coul2;
  o->rminl_coul2 = s->rminl_coul2;
  o->rmaxl_coul2 = s->rmaxl_coul2;
  o->rmaxs_skin2_e = s->rmaxs_skin2_e;
  o->rmaxl_skin2_e = s->rmaxl_skin2_e;
  o->excl_off = (int *)dup(s->excl_off, (n + 1) * 4.);
  o->excl_idx = (int *)dup(s->excl_idx, s->excl_off[n] * 4.);
  o->cexcl_off = (int *)dup(s->cexcl_off, (n + 1) * 4.);
  o->cexcl_idx = (int *)dup(s->cexcl_idx, s->cexcl_off[n] * 4.);
  /* icharge: set_charges elec_ngbr.c:115-121 */
  o->icharge = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  for (i = 0; i < n; i++)
    if (o->qch[i] != 0.) o->icharge[o->ncharge++] = i;
  o->ktot = s->ktot;
  o->ka = (int *)dup(s->ka, s->ktot * 4.);
  o->kb = (int *)dup(s->kb, s->ktot * 4.);
  o->kc = (int *)dup(s->kc, s->ktot * 4.);
  /* kup: first vector of every (ka, kb) row (ewald_setup md_ewald.c:95,102) */
  o->kup = (int *)calloc((size_t)s->ktot + 1, sizeof(int));
  for (i = 0; i < s->ktot; i++)
    o->kup[i] = (i == 0 || o->ka[i] != o->ka[i - 1] || o->kb[i] != o->kb[i - 1]);
  o->kappa = s->kappa;
  o->kappa2 = s->kappa * s->kappa;
  o->falp2 = s->falp2;
  o->ewald_self = s->ewald_self;
  o->ewald_bkg = s->ewald_bkg;
  o->necorr = s->necorr;
  o->iecorr = (int *)dup(s->iecorr, s->necorr * 4.);
  o->jecorr = (int *)dup(s->jecorr, s->necorr * 4.);
  o->nbonds = s->nbonds;
  o->ibond = (int *)dup(s->ibond, s->nbonds * 4.);
  o->jbond = (int *)dup(s->jbond, s->nbonds * 4.);
  o->idxbond = (int *)dup(s->idxbond, s->nbonds * 4.);
  o->itypbond = (int *)dup(s->itypbond, s->nbond_types * 4.);
  o->eqbond = (double *)dup(s->eqbond, s->nbond_types * 8.);
  o->fkbond = (double *)dup(s->fkbond, s->nbond_types * 8.);
  o->nbends = s->nbends;
  o->ibend = (int *)dup(s->ibend, s->nbends * 4.);
  o->jbend = (int *)dup(s->jbend, s->nbends * 4.);
  o->kbend = (int *)dup(s->kbend, s->nbends * 4.);
  o->idxbend = (int *)dup(s->idxbend, s->nbends * 4.);
  o->itypbend = (int *)dup(s->itypbend, s->nbend_types * 4.);
  o->eqbend = (double *)dup(s->eqbend, s->nbend_types * 8.);
  o->fkbend = (double *)dup(s->fkbend, s->nbend_types * 8.);
  o->ntors = s->ntors;
  if (s->ntors > 0) {
    o->itors = (int *)dup(s->itors, s->ntors * 4.);
    o->jtors = (int *)dup(s->jtors, s->ntors * 4.);
    o->ktors = (int *)dup(s->ktors, s->ntors * 4.);
    o->ltors = (int *)dup(s->ltors, s->ntors * 4.);
    o->idxtors = (int *)dup(s->idxtors, s->ntors * 4.);
    o->tors_form = (int *)dup(s->tors_ind_pot, s->ntors_types * 4.);
    o->tors_row = (int *)dup(s->tors_ind_pot_num, s->ntors_types * 4.);
    o->eqtors = (double *)dup(s->eqtors, s->ntors_harm * 8.);
    o->fktors = (double *)dup(s->fktors, s->ntors_harm * 8.);
    o->vphi = (double *)dup(s->vphi, (double)s->ntors_series * CM3D_NB_MAXPOWER_TORS * 8.);
  }
  o->n14 = s->n14;
  if (s->n14 > 0) {
    o->n14table = s->n14table;
    o->i14 = (int *)dup(s->i14, s->n14 * 4.);
    o->j14 = (int *)dup(s->j14, s->n14 * 4.);
    o->i14dx = (int *)dup(s->i14dx, s->n14 * 4.);
    o->r14min2 = (double *)dup(s->r14min2, s->n14_types * 8.);
    o->r14max2 = (double *)dup(s->r14max2, s->n14_types * 8.);
    o->dx214tab = (double *)dup(s->dx214tab, s->n14_types * 8.);
    o->v14tab = (double *)dup(s->v14tab, (double)s->n14_types * s->n14table * 8.);
    o->dv14tab = (double *)dup(s->dv14tab, (double)s->n14_types * s->n14table * 8.);
    o->scale14 = s->scale_onefour;
    o->scale14e = s->scale_onefour_e;
  }
  o->nbondx = s->nbondx;
  if (s->nbondx > 0) {
    o->ibondx = (int *)dup(s->ibondx, s->nbondx * 4.);
    o->jbondx = (int *)dup(s->jbondx, s->nbondx * 4.);
    o->kbondx = (int *)dup(s->kbondx, s->nbondx * 4.);
    o->idxbondx = (int *)dup(s->idxbondx, s->nbondx * 4.);
    o->eq1bondx = (double *)dup(s->eq1bondx, s->nbondx_types * 8.);
    o->eq2bondx = (double *)dup(s->eq2bondx, s->nbondx_types * 8.);
    o->fkbondx = (double *)dup(s->fkbondx, s->nbondx_types * 8.);
  }
  o->fxr = (double *)calloc(3 * (size_t)n + 1, 8);
  o->nfreeze = s->nfreeze;
  o->ifreeze = (int *)dup(s->ifreeze, s->nfreeze * 4.);
  o->ntherm = s->ntherm;
  o->nchain = s->nchain;
  if (s->ntherm > 0) {
    size_t tc = (size_t)s->ntherm * s->nchain;
    o->ithm = (int *)dup(s->ithm, n * 4.);
    o->mnh = (double *)dup(s->mnh, tc * 8.);
    o->gkt = (double *)dup(s->gkt, tc * 8.);
    o->eta = (double *)dup(s->nhc_eta, tc * 8.);
    o->veta = (double *)dup(s->nhc_veta, tc * 8.);
    o->feta = (double *)calloc(tc, 8);
    o->p2mt = (double *)calloc((size_t)s->ntherm, 8);
  }
  o->fxl = (double *)calloc(3 * (size_t)n + 1, 8);
  o->fxs = (double *)calloc(3 * (size_t)n + 1, 8);
  o->fxa = (double *)calloc(3 * (size_t)n + 1, 8);
  o->scr = (double *)calloc(3 * (size_t)n + 1, 8);
  o->rec = (double *)calloc(3 * (size_t)n + 1, 8);
  o->dxn = (double *)calloc(3 * (size_t)n + 1, 8);
  o->lnk = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  o->hlist = (int *)malloc(sizeof(int) * (size_t)ncells * ncells * ncells);
  return o;
}

void orc_destroy(orc *o)
{
  void *ptrs[] = {o->px, o->py, o->pz, o->vx, o->vy, o->vz, o->amass, o->qch,
                  o->itype, o->map, o->vtab, o->dvtab, o->switchs, o->rmaxs_cut2,
                  o->rmins_cut2, o->rmaxl_cut2, o->rminl_cut2, o->rmaxs_skin2,
                  o->rmaxl_skin2, o->dx2tab, o->coultab, o->dcoultab, o->switchse,
                  o->excl_off, o->excl_idx, o->cexcl_off, o->cexcl_idx, o->icharge,
                  o->ka, o->kb, o->kc, o->kup, o->iecorr, o->jecorr, o->ibond,
                  o->jbond, o->idxbond, o->itypbond, o->eqbond, o->fkbond, o->ibend,
                  o->jbend, o->kbend, o->idxbend, o->itypbend, o->eqbend, o->fkbend,
                  o->fxl, o->fxs, o->fxa, o->scr, o->rec, o->dxn, o->inpt, o->jnpt,
                  o->inps, o->jnps, o->inpte, o->jnpte, o->inpse, o->jnpse, o->icell,
                  o->jcell, o->icelle, o->jcelle, o->hlist, o->lnk, o->itors, o->jtors,
                  o->ktors, o->ltors, o->idxtors, o->tors_form, o->tors_row, o->eqtors,
                  o->fktors, o->vphi, o->i14, o->j14, o->i14dx, o->r14min2, o->r14max2,
                  o->dx214tab, o->v14tab, o->dv14tab, o->ibondx, o->jbondx, o->kbondx,
                  o->idxbondx, o->eq1bondx, o->eq2bondx, o->fkbondx, o->fxr, o->ifreeze,
                  o->ithm, o->mnh, o->gkt, o->eta, o->veta, o->feta, o->p2mt};
  size_t i;
  for (i = 0; i < sizeof ptrs / sizeof ptrs[0]; i++) free(ptrs[i]);
  free(o);
}

void orc_set_positions(orc *o, const double *px, const double *py, const double *pz)
{
  memcpy(o->px, px, o->n * 8.);
  memcpy(o->py, py, o->n * 8.);
  memcpy(o->pz, pz, o->n * 8.);
}
void orc_get_positions(orc *o, double *px, double *py, double *pz)
{
  memcpy(px, o->px, o->n * 8.);
  memcpy(py, o->py, o->n * 8.);
  memcpy(pz, o->pz, o->n * 8.);
}
void orc_set_velocities(orc *o, const double *vx, const double *vy, const double *vz)
{
  memcpy(o->vx, vx, o->n * 8.);
  memcpy(o->vy, vy, o->n * 8.);
  memcpy(o->vz, vz, o->n * 8.);
}
void orc_get_velocities(orc *o, double *vx, double *vy, double *vz)
{
  memcpy(vx, o->vx, o->n * 8.);
  memcpy(vy, o->vy, o->n * 8.);
  memcpy(vz, o->vz, o->n * 8.);
}
static double *block(orc *o, int which)
{
  return which == 0 ? o->fxl : which == 1 ? o->fxs : which == 2 ? o->fxa : o->fxr;
}
void orc_get_forces(orc *o, int which, double *fx, double *fy, double *fz)
{
  double *b = block(o, which);
  memcpy(fx, b, o->n * 8.);
  memcpy(fy, b + o->n, o->n * 8.);
  memcpy(fz, b + 2 * o->n, o->n * 8.);
}
void orc_zero_forces(orc *o, int which)
{
  memset(block(o, which), 0, 3 * (size_t)o->n * 8);
}

/* ------------------------------------------------------------ link cells */
/* set_link  energy/control/set_link.c:31-201: half-shell cell pairs whose
   (conservative) separation is below rmax (LJ) / rmaxe (charges) */
static void set_link(orc *o, double rmax, double rmaxe)
{
  const double *h = o->hmat;
  int ncell = o->ncells, nmax = ncell / 2, ncell2 = ncell * ncell;
  int ncells = ncell * ncell2, icell, ic, jc, kc, i, j, k, in, jn, kn, cap;
  double rcell = 1. / (double)ncell, ddot, sinangle, dx, dy, dz, r;
  free(o->icell); free(o->jcell); free(o->icelle); free(o->jcelle);
  cap = ncells * (nmax + 1) * (2 * nmax + 1) * (2 * nmax + 1) + 1;
  o->icell = (int *)malloc(sizeof(int) * cap);
  o->jcell = (int *)malloc(sizeof(int) * cap);
  o->icelle = (int *)malloc(sizeof(int) * cap);
  o->jcelle = (int *)malloc(sizeof(int) * cap);
  o->npaircell = o->npaircelle = 0;
  ddot = h[0] * h[3] + h[1] * h[4] + h[2] * h[5];
  ddot /= (sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]) * sqrt(h[3] * h[3] + h[4] * h[4] + h[5] * h[5]));
  sinangle = sin(acos(ddot));
  ddot = h[0] * h[6] + h[1] * h[7] + h[2] * h[8];
  ddot /= (sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]) * sqrt(h[6] * h[6] + h[7] * h[7] + h[8] * h[8]));
  ddot = sin(acos(ddot));
  if (ddot < sinangle) sinangle = ddot;
  ddot = h[3] * h[6] + h[4] * h[7] + h[5] * h[8];
  ddot /= (sqrt(h[3] * h[3] + h[4] * h[4] + h[5] * h[5]) * sqrt(h[6] * h[6] + h[7] * h[7] + h[8] * h[8]));
  ddot = sin(acos(ddot));
  if (ddot < sinangle) sinangle = ddot;
  for (icell = 0; icell < ncells; icell++) {
    ic = icell / ncell2;
    jc = (icell - ic * ncell2) / ncell;
    kc = (icell - ic * ncell2 - jc * ncell);
    for (i = 0; i <= nmax; i++) {
      for (j = (i == 0) ? 0 : -nmax; j <= nmax; j++) {
        for (k = (i == 0 && j == 0) ? 0 : -nmax; k <= nmax; k++) {
          in = (ic + i) % ncell;
          jn = (jc + j) % ncell;
          kn = (kc + k) % ncell;
          in = abs(ic - in);
          jn = abs(jc - jn);
          kn = abs(kc - kn);
          if (o->iperd > 0 && in > ncell / 2) in = ncell - in;
          if (o->iperd > 1 && jn > ncell / 2) jn = ncell - jn;
          if (o->iperd > 2 && kn > ncell / 2) kn = ncell - kn;
          if (in > 0) in--;
          if (jn > 0) jn--;
          if (kn > 0) kn--;
          dx = h[0] * in * rcell + h[1] * jn * rcell + h[2] * kn * rcell;
          dy = h[3] * in * rcell + h[4] * jn * rcell + h[5] * kn * rcell;
          dz = h[6] * in * rcell + h[7] * jn * rcell + h[8] * kn * rcell;
          r = sqrt(dx * dx + dy * dy + dz * dz) * sinangle;
          if (r < rmax || r < rmaxe) {
            in = ic + i; jn = jc + j; kn = kc + k;
            if (in < 0) in += ncell;
            if (jn < 0) jn += ncell;
            if (kn < 0) kn += ncell;
            if (in >= ncell) in -= ncell;
            if (jn >= ncell) jn -= ncell;
            if (kn >= ncell) kn -= ncell;
            if (r < rmax) {
              o->icell[o->npaircell] = icell;
              o->jcell[o->npaircell++] = in * ncell2 + jn * ncell + kn;
            }
            if (r < rmaxe) {
              o->icelle[o->npaircelle] = icell;
              o->jcelle[o->npaircelle++] = in * ncell2 + jn * ncell + kn;
            }
          }
        }
      }
    }
  }
  o->cells_ready = 1;
}

/* get_lnklist / get_lnklist_e  set_link.c:203-300: chains built from the last
   atom down so that every chain is in ascending atom order; only charged
   atoms when `charged_only` */
static void get_lnklist(orc *o, int charged_only)
{
  int ncell = o->ncells, ncell2 = ncell * ncell, ncell3 = ncell * ncell2;
  int ncellm1 = ncell - 1, i, ic, jc, kc, icell;
  double hi[9];
  gethinv9(o->hmat, hi);
  for (i = 0; i < ncell3; i++) o->hlist[i] = -1;
  for (i = o->n - 1; i >= 0; i--) {
    double sx, sy, sz;
    if (charged_only && o->qch[i] == 0.0) continue;
    sx = o->px[i] * hi[0] + o->py[i] * hi[1] + o->pz[i] * hi[2];
    sy = o->px[i] * hi[3] + o->py[i] * hi[4] + o->pz[i] * hi[5];
    sz = o->px[i] * hi[6] + o->py[i] * hi[7] + o->pz[i] * hi[8];
    if (o->iperd > 0) sx -= ANINT(sx);
    if (o->iperd > 1) sy -= ANINT(sy);
    if (o->iperd > 2) sz -= ANINT(sz);
    ic = (int)((sx + .5) * ncell);
    jc = (int)((sy + .5) * ncell);
    kc = (int)((sz + .5) * ncell);
    ic = ic > 0 ? ic : 0; jc = jc > 0 ? jc : 0; kc = kc > 0 ? kc : 0;
    ic = ic < ncellm1 ? ic : ncellm1;
    jc = jc < ncellm1 ? jc : ncellm1;
    kc = kc < ncellm1 ? kc : ncellm1;
    icell = ic * ncell2 + jc * ncell + kc;
    o->lnk[i] = o->hlist[icell];
    o->hlist[icell] = i;
  }
}

/* ------------------------------------------------------ Verlet lists */
static void push(int **ip, int **jp, long long *np, long long *cap, int i, int j)
{
  if (*np >= *cap) {
    *cap = *cap ? 2 * *cap : 1024;
    *ip = (int *)realloc(*ip, sizeof(int) * (size_t)*cap);
    *jp = (int *)realloc(*jp, sizeof(int) * (size_t)*cap);
  }
  (*ip)[*np] = i;
  (*jp)[*np] = j;
  (*np)++;
}

/* candidate test of ngbr_list  ngbr_list.c:60-97: min-image r^2 against the
   per-interaction skin radii (t list; s list nested inside) */
static void test_lj(orc *o, int in, int jn)
{
  double xd = o->px[in] - o->px[jn], yd = o->py[in] - o->py[jn], zd = o->pz[in] - o->pz[jn];
  double r2;
  int intr;
  period(1, &xd, &yd, &zd, o->hmat, o->hmati);
  r2 = xd * xd + yd * yd + zd * zd;
  intr = o->map[o->itype[in] * o->ntypes + o->itype[jn]];
  if (r2 < o->rmaxl_skin2[intr]) {
    push(&o->inpt, &o->jnpt, &o->nprt, &o->cap_t, in, jn);
    if (r2 < o->rmaxs_skin2[intr]) push(&o->inps, &o->jnps, &o->nprs, &o->cap_s, in, jn);
  }
}

/* ngbr_liste  ngbr_list.c:114-140 */
static void test_el(orc *o, int in, int jn)
{
  double xd = o->px[in] - o->px[jn], yd = o->py[in] - o->py[jn], zd = o->pz[in] - o->pz[jn];
  double r2;
  period(1, &xd, &yd, &zd, o->hmat, o->hmati);
  r2 = xd * xd + yd * yd + zd * zd;
  if (r2 < o->rmaxl_skin2_e) {
    push(&o->inpte, &o->jnpte, &o->nprte, &o->cap_te, in, jn);
    if (r2 < o->rmaxs_skin2_e) push(&o->inpse, &o->jnpse, &o->nprse, &o->cap_se, in, jn);
  }
}

/* get_ngbr  ngbr_list.c:297-581 and get_ngbr_e  elec_ngbr.c:220-358 */
void orc_get_ngbr(orc *o)
{
  int n = o->n, i, j, p;
  gethinv9(o->hmat, o->hmati);
  o->nprt = o->nprs = o->nprte = o->nprse = 0;
  if (!o->cells_ready && o->nocell_all) {
    double r2 = 0;
    for (i = 0; i < o->ninter; i++)
      if (o->rmaxl_skin2[i] > r2) r2 = o->rmaxl_skin2[i];
    set_link(o, sqrt(r2) + o->skin, sqrt(o->rmaxl_skin2_e) + o->skin);
  }
  /* LJ lists */
  if (o->nocell_all == 0) {
    for (i = 0; i < n; i++)
      for (j = i + 1; j < n; j++) {
        if (exclij(i, j, o->excl_off, o->excl_idx)) continue;
        if (o->map[o->itype[i] * o->ntypes + o->itype[j]] == -1) continue;
        test_lj(o, i, j);
      }
  } else {
    get_lnklist(o, 0);
    for (p = 0; p < o->npaircell; p++) {
      int icell = o->icell[p], jcell = o->jcell[p];
      int ii = o->hlist[icell];
      while (ii != -1) {
        int jj = (icell == jcell) ? o->lnk[ii] : o->hlist[jcell];
        while (jj != -1) {
          if (o->map[o->itype[ii] * o->ntypes + o->itype[jj]] != -1 &&
              !exclij(ii, jj, o->excl_off, o->excl_idx))
            test_lj(o, ii, jj);
          jj = o->lnk[jj];
        }
        ii = o->lnk[ii];
      }
    }
  }
  /* charged lists */
  if (o->ncharge > 0) {
    if (o->nocell_all == 0) {
      for (i = 0; i < o->ncharge; i++)
        for (j = i + 1; j < o->ncharge; j++) {
          int ii = o->icharge[i], jj = o->icharge[j];
          if (exclij(ii, jj, o->cexcl_off, o->cexcl_idx)) continue;
          test_el(o, ii, jj);
        }
    } else {
      get_lnklist(o, 1);
      for (p = 0; p < o->npaircelle; p++) {
        int icell = o->icelle[p], jcell = o->jcelle[p];
        int ii = o->hlist[icell];
        while (ii != -1) {
          int jj = (icell == jcell) ? o->lnk[ii] : o->hlist[jcell];
          while (jj != -1) {
            if (!exclij(ii, jj, o->cexcl_off, o->cexcl_idx)) test_el(o, ii, jj);
            jj = o->lnk[jj];
          }
          ii = o->lnk[ii];
        }
      }
    }
  }
  /* positions snapshot  ngbr_list.c:577-580 */
  memcpy(o->dxn, o->px, n * 8.);
  memcpy(o->dxn + n, o->py, n * 8.);
  memcpy(o->dxn + 2 * n, o->pz, n * 8.);
  o->rebuilds++;
}

long long orc_list_count(orc *o, int which)
{
  return which == 0 ? o->nprt : which == 1 ? o->nprs : which == 2 ? o->nprte : o->nprse;
}
void orc_get_list(orc *o, int which, int *ip, int *jp)
{
  long long n = orc_list_count(o, which);
  int *a = which == 0 ? o->inpt : which == 1 ? o->inps : which == 2 ? o->inpte : o->inpse;
  int *b = which == 0 ? o->jnpt : which == 1 ? o->jnps : which == 2 ? o->jnpte : o->jnpse;
  if (n > 0) {
    memcpy(ip, a, sizeof(int) * (size_t)n);
    memcpy(jp, b, sizeof(int) * (size_t)n);
  }
}

/* ------------------------------------------------------- pair kernels */
/* 3-point table interpolation  md_fnopol.c:148 */
#define INTERP(t, k, p) ((t)[k] + .5 * (p) * ((t)[(k) + 1] - (t)[(k) - 1] + (p) * ((t)[(k) - 1] - 2. * (t)[k] + (t)[(k) + 1])))

/* force_npol  energy/inter/md_fnopol.c:46-255 over one chunk */
static void force_npol(orc *o, int nlen, const int *indx, const int *jndx, int iflg)
{
  int n = o->n, n2 = 2 * n, j;
  const double *rmax2 = iflg == 0 ? o->rmaxs_cut2 : o->rmaxl_cut2;
  double spotlt = 0., spothlt = 0.;
  double *xd = (double *)malloc(6 * sizeof(double) * (size_t)(nlen > 0 ? nlen : 1));
  double *yd = xd + nlen, *zd = xd + 2 * nlen, *fxd = xd + 3 * nlen, *fyd = xd + 4 * nlen,
         *fzd = xd + 5 * nlen;
  int ntm4 = o->ntable - 4;
  double hi[9];
  gethinv9(o->hmat, hi);
  for (j = 0; j < nlen; j++) {
    xd[j] = o->px[indx[j]] - o->px[jndx[j]];
    yd[j] = o->py[indx[j]] - o->py[jndx[j]];
    zd[j] = o->pz[indx[j]] - o->pz[jndx[j]];
  }
  period(nlen, xd, yd, zd, o->hmat, hi);
  for (j = 0; j < nlen; j++) {
    int in = o->map[o->itype[indx[j]] * o->ntypes + o->itype[jndx[j]]];
    double dis2 = xd[j] * xd[j] + yd[j] * yd[j] + zd[j] * zd[j];
    if (dis2 < rmax2[in]) {
      double p = (dis2 - o->rmins_cut2[in]) * o->dx2tab[in], f, swv;
      int k = (int)p;
      const double *t = o->dvtab + (size_t)in * o->ntable;
      if (k < 1) {
        o->underflows++;
        k = 1;
        p = 1.;
      }
      p = p - (double)k;
      f = INTERP(t, k, p);
      if (dis2 > o->rminl_cut2[in]) {
        const double *sw = o->switchs + (size_t)in * o->ntable;
        swv = INTERP(sw, k, p);
      } else {
        swv = 1.;
      }
      if (iflg == 1) {
        const double *vt = o->vtab + (size_t)in * o->ntable;
        double fcc;
        o->sprsl -= dis2 * f;
        o->sprslt[0] -= xd[j] * xd[j] * f;
        o->sprslt[1] -= yd[j] * xd[j] * f;
        o->sprslt[2] -= zd[j] * xd[j] * f;
        o->sprslt[4] -= yd[j] * yd[j] * f;
        o->sprslt[5] -= zd[j] * yd[j] * f;
        o->sprslt[8] -= zd[j] * zd[j] * f;
        xd[j] *= f;
        yd[j] *= f;
        zd[j] *= f;
        fxd[j] = xd[j] * swv;
        fyd[j] = yd[j] * swv;
        fzd[j] = zd[j] * swv;
        fcc = INTERP(vt, k, p);
        spotlt += fcc;
        spothlt += fcc - vt[ntm4];
      } else {
        f *= swv;
        xd[j] *= f;
        yd[j] *= f;
        zd[j] *= f;
      }
    } else {
      xd[j] = yd[j] = zd[j] = 0.;
      fxd[j] = fyd[j] = fzd[j] = 0.;
    }
  }
  if (iflg == 1) {
    o->sprslt[3] = o->sprslt[1];
    o->sprslt[6] = o->sprslt[2];
    o->sprslt[7] = o->sprslt[5];
  }
  o->spotl += spotlt;
  o->spothl += spothlt;
  for (j = 0; j < nlen; j++) {
    int ni = indx[j], nj = jndx[j];
    o->scr[ni] -= xd[j];
    o->scr[ni + n] -= yd[j];
    o->scr[ni + n2] -= zd[j];
    o->scr[nj] += xd[j];
    o->scr[nj + n] += yd[j];
    o->scr[nj + n2] += zd[j];
    if (iflg == 1) {
      o->rec[ni] -= fxd[j];
      o->rec[ni + n] -= fyd[j];
      o->rec[ni + n2] -= fzd[j];
      o->rec[nj] += fxd[j];
      o->rec[nj + n] += fyd[j];
      o->rec[nj + n2] += fzd[j];
    }
  }
  free(xd);
}

/* force_ter  energy/control/md_finter.c:110-310 (verlist branch) */
void orc_force_ter(orc *o, int iflg)
{
  int n3 = 3 * o->n, i;
  long long np = iflg == 0 ? o->nprs : o->nprt, s;
  const int *ip = iflg == 0 ? o->inps : o->inpt, *jp = iflg == 0 ? o->jnps : o->jnpt;
  double *fx = iflg == 0 ? o->fxs : o->fxl;
  if (iflg == 1) {
    o->spotl = o->spothl = o->sprsl = 0.;
    for (i = 0; i < 9; i++) o->sprslt[i] = 0.;
    for (i = 0; i < n3; i++) o->scr[i] = o->rec[i] = 0.;
  } else {
    for (i = 0; i < n3; i++) o->scr[i] = 0.;
  }
  for (s = 0; s < np; s += o->nlen) {
    int k = (int)(np - s < o->nlen ? np - s : o->nlen);
    force_npol(o, k, ip + s, jp + s, iflg);
  }
  for (i = 0; i < n3; i++) fx[i] += o->scr[i];
  if (iflg == 1)
    for (i = 0; i < n3; i++) o->fxs[i] += o->rec[i];
}

/* force_e  energy/inter/finter_e.c:42-233 over one chunk; note the
   fall-through of its switch (finter_e.c:72-83): both levels use the full
   rmaxl_coul2 cutoff and the switch never engages */
static void force_e(orc *o, int nlen, const int *indx, const int *jndx, int iflg)
{
  int n = o->n, n2 = 2 * n, j, ntable = o->ntable;
  double rmax2 = o->rmaxl_coul2, rmin2 = o->rmaxl_coul2, tablast = o->coultab[ntable - 4];
  double sphet = 0., spet = 0.;
  double *xd = (double *)malloc(10 * sizeof(double) * (size_t)(nlen > 0 ? nlen : 1));
  double *yd = xd + nlen, *zd = xd + 2 * nlen, *fxd = xd + 3 * nlen, *fyd = xd + 4 * nlen,
         *fzd = xd + 5 * nlen, *qij = xd + 6 * nlen, *fx = xd + 7 * nlen, *fy = xd + 8 * nlen,
         *fz = xd + 9 * nlen;
  double hi[9];
  gethinv9(o->hmat, hi);
  for (j = 0; j < nlen; j++) {
    xd[j] = o->px[indx[j]] - o->px[jndx[j]];
    yd[j] = o->py[indx[j]] - o->py[jndx[j]];
    zd[j] = o->pz[indx[j]] - o->pz[jndx[j]];
    qij[j] = o->qch[indx[j]] * o->qch[jndx[j]];
  }
  period(nlen, xd, yd, zd, o->hmat, hi);
  for (j = 0; j < nlen; j++) {
    double dis2 = xd[j] * xd[j] + yd[j] * yd[j] + zd[j] * zd[j];
    if (dis2 < rmax2) {
      double p = (dis2 - o->rmins_coul2) * o->dx2coul, f, swv, fcc, q;
      int k = (int)p;
      if (k < 1) {
        o->underflows++;
        k = 1;
        p = 1;
      }
      p = p - (double)k;
      f = INTERP(o->dcoultab, k, p);
      if (dis2 > rmin2) swv = INTERP(o->switchse, k, p);
      else swv = 1.;
      q = qij[j];
      fcc = q * f;
      if (iflg == 1) {
        o->sprse -= dis2 * fcc;
        o->sprset[0] -= xd[j] * xd[j] * fcc;
        o->sprset[1] -= yd[j] * xd[j] * fcc;
        o->sprset[2] -= zd[j] * xd[j] * fcc;
        o->sprset[4] -= yd[j] * yd[j] * fcc;
        o->sprset[5] -= zd[j] * yd[j] * fcc;
        o->sprset[8] -= zd[j] * zd[j] * fcc;
        fx[j] = xd[j] * fcc;
        fy[j] = yd[j] * fcc;
        fz[j] = zd[j] * fcc;
        fxd[j] = fx[j] * swv;
        fyd[j] = fy[j] * swv;
        fzd[j] = fz[j] * swv;
        f = INTERP(o->coultab, k, p);
        sphet += q * (f - tablast);
        spet += q * f;
      } else {
        fcc *= swv;
        fx[j] = xd[j] * fcc;
        fy[j] = yd[j] * fcc;
        fz[j] = zd[j] * fcc;
      }
    } else {
      fx[j] = fy[j] = fz[j] = 0.;
      fxd[j] = fyd[j] = fzd[j] = 0.;
    }
  }
  o->spothe += sphet;
  o->spote += spet;
  if (iflg == 1) {
    o->sprset[3] = o->sprset[1];
    o->sprset[6] = o->sprset[2];
    o->sprset[7] = o->sprset[5];
  }
  for (j = 0; j < nlen; j++) {
    int ni = indx[j], nj = jndx[j];
    o->scr[ni] -= fx[j];
    o->scr[ni + n] -= fy[j];
    o->scr[ni + n2] -= fz[j];
    o->scr[nj] += fx[j];
    o->scr[nj + n] += fy[j];
    o->scr[nj + n2] += fz[j];
    if (iflg == 1) {
      o->rec[ni] -= fxd[j];
      o->rec[ni + n] -= fyd[j];
      o->rec[ni + n2] -= fzd[j];
      o->rec[nj] += fxd[j];
      o->rec[nj + n] += fyd[j];
      o->rec[nj + n2] += fzd[j];
    }
  }
  free(xd);
}

/* force_ter_e  energy/control/md_finter_e.c:78-233 (verlist branch) */
void orc_force_ter_e(orc *o, int iflg)
{
  int n3 = 3 * o->n, i;
  long long np = iflg == 0 ? o->nprse : o->nprte, s;
  const int *ip = iflg == 0 ? o->inpse : o->inpte, *jp = iflg == 0 ? o->jnpse : o->jnpte;
  double *fx = iflg == 0 ? o->fxs : o->fxl;
  for (i = 0; i < n3; i++) o->scr[i] = o->rec[i] = 0.;
  if (iflg == 1) {
    o->spothe = o->spote = o->sprse = 0.;
    for (i = 0; i < 9; i++) o->sprset[i] = 0.;
  }
  if (o->ncharge == 0) return;
  for (s = 0; s < np; s += o->nlen) {
    int k = (int)(np - s < o->nlen ? np - s : o->nlen);
    force_e(o, k, ip + s, jp + s, iflg);
  }
  for (i = 0; i < n3; i++) fx[i] += o->scr[i];
  if (iflg == 1)
    for (i = 0; i < n3; i++) o->fxs[i] += o->rec[i];
}

/* fk_ewald  energy/inter/md_ewald.c:185-361 (serial: one rank holds every k) */
void orc_fk_ewald(orc *o)
{
  int nq = o->ncharge, i, j, n = o->n;
  double fact = sqrt(4.0 * M_PI), hi[9], rvol, vk = 0., vp = 0., vpt[9] = {0};
  double *tx, *ty, *tz, *tq, *cossc, *sinsc, *helr, *heli, six;
  double *fx = o->fxl, *fy = o->fxl + n, *fz = o->fxl + 2 * n;
  rvol = 1. / gethinv9(o->hmat, hi);
  if (nq == 0 || o->ktot == 0) {
    o->vk_ewald = o->vp_ewald = 0.;
    memset(o->vp_ewald_tensor, 0, sizeof o->vp_ewald_tensor);
    return;
  }
  tx = (double *)malloc(8 * sizeof(double) * (size_t)nq);
  ty = tx + nq; tz = tx + 2 * nq; tq = tx + 3 * nq;
  cossc = tx + 4 * nq; sinsc = tx + 5 * nq; helr = tx + 6 * nq; heli = tx + 7 * nq;
  for (j = 0; j < nq; j++) {
    int jj = o->icharge[j];
    tx[j] = o->px[jj]; ty[j] = o->py[jj]; tz[j] = o->pz[jj];
    tq[j] = o->qch[jj] * fact;
  }
  for (j = 0; j < nq; j++) {
    double akc = (tx[j] * hi[6] + ty[j] * hi[7] + tz[j] * hi[8]) * TPI;
    cossc[j] = cos(akc);
    sinsc[j] = sin(akc);
  }
  for (i = 0; i < o->ktot; i++) {
    double sx = TPI * o->ka[i], sy = TPI * o->kb[i], sz = TPI * o->kc[i];
    double aka = (sx * hi[0] + sy * hi[3] + sz * hi[6]);
    double akb = (sx * hi[1] + sy * hi[4] + sz * hi[7]);
    double akc = (sx * hi[2] + sy * hi[5] + sz * hi[8]);
    double g2 = aka * aka + akb * akb + akc * akc;
    double preg = exp(-g2 * o->falp2) * rvol / g2;
    double prep = -2. * preg * (g2 * o->falp2 + 1.) / g2;
    double sumr, sumi, smag;
    if (o->kup[i] || i == 0) {
      for (j = 0; j < nq; j++) {
        double rk = (tx[j] * aka + ty[j] * akb + tz[j] * akc);
        helr[j] = cos(rk);
        heli[j] = sin(rk);
      }
    } else {
      for (j = 0; j < nq; j++) {
        double rhr = helr[j], rhi = heli[j];
        sumr = cossc[j];
        sumi = sinsc[j];
        helr[j] = rhr * sumr - rhi * sumi;
        heli[j] = rhi * sumr + rhr * sumi;
      }
    }
    sumr = sumi = 0.;
    for (j = 0; j < nq; j++) {
      sumr += tq[j] * helr[j];
      sumi += tq[j] * heli[j];
    }
    smag = sumr * sumr + sumi * sumi;
    vk += preg * smag;
    vp += prep * smag * g2;
    vpt[0] += prep * smag * aka * aka;
    vpt[1] += prep * smag * akb * aka;
    vpt[2] += prep * smag * akc * aka;
    vpt[3] += prep * smag * aka * akb;
    vpt[4] += prep * smag * akb * akb;
    vpt[5] += prep * smag * akc * akb;
    vpt[6] += prep * smag * aka * akc;
    vpt[7] += prep * smag * akb * akc;
    vpt[8] += prep * smag * akc * akc;
    sumr *= 2. * preg;
    sumi *= 2. * preg;
    for (j = 0; j < nq; j++) {
      int jj = o->icharge[j];
      double q = tq[j], rhr = helr[j], rhi = heli[j];
      double srx = aka * sumr * q, sry = akb * sumr * q, srz = akc * sumr * q;
      double sxi = aka * sumi * q, syi = akb * sumi * q, szi = akc * sumi * q;
      fx[jj] += srx * rhi - sxi * rhr;
      fy[jj] += sry * rhi - syi * rhr;
      fz[jj] += srz * rhi - szi * rhr;
    }
  }
  six = o->ewald_bkg / get_deth(o->hmat);
  o->vk_ewald = vk + six + o->ewald_self;
  o->vp_ewald = vp + 3. * (vk + six);
  for (i = 0; i < 9; i++) o->vp_ewald_tensor[i] = vpt[i];
  o->vp_ewald_tensor[0] += vk + six;
  o->vp_ewald_tensor[4] += vk + six;
  o->vp_ewald_tensor[8] += vk + six;
  free(tx);
}

/* ecorr  energy/inter/md_ewald.c:385-453 (no minimum image, as in CM3D) */
void orc_ecorr(orc *o)
{
  int i, n = o->n;
  double spot = 0., sprs = 0., st[9] = {0}, sqrt_pi = 1. / sqrt(M_PI);
  double *fx = o->fxl, *fy = o->fxl + n, *fz = o->fxl + 2 * n;
  for (i = 0; i < o->necorr; i++) {
    int ii = o->iecorr[i], jj = o->jecorr[i];
    double xd = o->px[ii] - o->px[jj], yd = o->py[ii] - o->py[jj], zd = o->pz[ii] - o->pz[jj];
    double dis2 = xd * xd + yd * yd + zd * zd, dis = sqrt(dis2);
    double qijr = o->qch[ii] * o->qch[jj] / dis, ralp = dis * o->kappa, erfr = erf(ralp), dv;
    spot += -qijr * erfr;
    dv = -qijr * (-2. * o->kappa * exp(-o->kappa2 * dis2) * sqrt_pi + erfr / dis);
    sprs += dis * dv;
    dv /= dis;
    st[0] += dv * xd * xd; st[1] += dv * xd * yd; st[2] += dv * xd * zd;
    st[3] += dv * yd * xd; st[4] += dv * yd * yd; st[5] += dv * yd * zd;
    st[6] += dv * zd * xd; st[7] += dv * zd * yd; st[8] += dv * zd * zd;
    xd *= dv; yd *= dv; zd *= dv;
    fx[ii] += xd; fy[ii] += yd; fz[ii] += zd;
    fx[jj] -= xd; fy[jj] -= yd; fz[jj] -= zd;
  }
  o->pot_ecorr = spot;
  o->prs_ecorr = sprs;
  memcpy(o->prs_ecorr_tensor, st, sizeof st);
}

/* fbond  energy/intra/md_fbond.c:76-125 (harmonic) */
void orc_fbond(orc *o)
{
  int nb, n = o->n;
  double *fx = o->fxa, *fy = o->fxa + n, *fz = o->fxa + 2 * n;
  for (nb = 0; nb < o->nbonds; nb++) {
    int i = o->ibond[nb], j = o->jbond[nb], idx = o->idxbond[nb];
    double dx = o->px[i] - o->px[j], dy = o->py[i] - o->py[j], dz = o->pz[i] - o->pz[j];
    double r = sqrt(dx * dx + dy * dy + dz * dz), dr = r - o->eqbond[idx];
    double fr = o->fkbond[idx] * dr / r;
    dx *= fr; dy *= fr; dz *= fr;
    fx[i] -= dx; fy[i] -= dy; fz[i] -= dz;
    fx[j] += dx; fy[j] += dy; fz[j] += dz;
  }
}

/* fbend  energy/intra/md_fbend.c:126-260 (harmonic) */
void orc_fbend(orc *o)
{
  int nb, n = o->n;
  double *fx = o->fxa, *fy = o->fxa + n, *fz = o->fxa + 2 * n;
  double *f9 = (double *)malloc(9 * sizeof(double) * (size_t)(o->nbends > 0 ? o->nbends : 1));
  for (nb = 0; nb < o->nbends; nb++) {
    int i = o->ibend[nb], j = o->jbend[nb], k = o->kbend[nb], idx = o->idxbend[nb];
    double ax = o->px[i] - o->px[j], ay = o->py[i] - o->py[j], az = o->pz[i] - o->pz[j];
    double al = ax * ax + ay * ay + az * az;
    double bx = o->px[k] - o->px[j], by = o->py[k] - o->py[j], bz = o->pz[k] - o->pz[j];
    double bl = bx * bx + by * by + bz * bz;
    double adotb = ax * bx + ay * by + az * bz;
    double r11 = 1. / sqrt(al * bl), costh = adotb * r11, th, dth, dudth, dthdcos, dudcos;
    double d1x, d1y, d1z, d3x, d3y, d3z;
    if (fabs(costh) >= 1.) {
      dthdcos = -1.;
      dudth = 0.;
    } else {
      th = acos(costh);
      dth = th - o->eqbend[idx];
      dudth = o->fkbend[idx] * dth;
      dthdcos = -1. / sqrt(1. - costh * costh);
    }
    dudcos = dudth * dthdcos;
    d1x = costh * ax / al - bx * r11;
    d1y = costh * ay / al - by * r11;
    d1z = costh * az / al - bz * r11;
    d3x = costh * bx / bl - ax * r11;
    d3y = costh * by / bl - ay * r11;
    d3z = costh * bz / bl - az * r11;
    f9[9 * nb + 0] = dudcos * d1x;
    f9[9 * nb + 1] = dudcos * d1y;
    f9[9 * nb + 2] = dudcos * d1z;
    f9[9 * nb + 3] = dudcos * (-d1x - d3x);
    f9[9 * nb + 4] = dudcos * (-d1y - d3y);
    f9[9 * nb + 5] = dudcos * (-d1z - d3z);
    f9[9 * nb + 6] = dudcos * d3x;
    f9[9 * nb + 7] = dudcos * d3y;
    f9[9 * nb + 8] = dudcos * d3z;
  }
  for (nb = 0; nb < o->nbends; nb++) {
    int i = o->ibend[nb], j = o->jbend[nb], k = o->kbend[nb];
    fx[i] += f9[9 * nb + 0]; fy[i] += f9[9 * nb + 1]; fz[i] += f9[9 * nb + 2];
    fx[j] += f9[9 * nb + 3]; fy[j] += f9[9 * nb + 4]; fz[j] += f9[9 * nb + 5];
    fx[k] += f9[9 * nb + 6]; fy[k] += f9[9 * nb + 7]; fz[k] += f9[9 * nb + 8];
  }
  free(f9);
}

/* fbondx  energy/intra/md_fbocross.c:40-97: the cross (bond-bond) term
   fk (|ri - rj| - eq1)(|rj - rk| - eq2) */
void orc_fbondx(orc *o)
{
  int nb, n = o->n;
  double *fx = o->fxa, *fy = o->fxa + n, *fz = o->fxa + 2 * n;
  for (nb = 0; nb < o->nbondx; nb++) {
    int i = o->ibondx[nb], j = o->jbondx[nb], k = o->kbondx[nb], t = o->idxbondx[nb];
    double ax = o->px[i] - o->px[j], ay = o->py[i] - o->py[j], az = o->pz[i] - o->pz[j];
    double al = sqrt(ax * ax + ay * ay + az * az);
    double bx = o->px[j] - o->px[k], by = o->py[j] - o->py[k], bz = o->pz[j] - o->pz[k];
    double bl = sqrt(bx * bx + by * by + bz * bz);
    double dr1 = al - o->eq1bondx[t], dr2 = bl - o->eq2bondx[t];
    double fr1 = o->fkbondx[t] * dr2 / al, fr2 = o->fkbondx[t] * dr1 / bl;
    fx[i] += -fr1 * ax; fy[i] += -fr1 * ay; fz[i] += -fr1 * az;
    fx[j] += fr1 * ax - fr2 * bx; fy[j] += fr1 * ay - fr2 * by; fz[j] += fr1 * az - fr2 * bz;
    fx[k] += fr2 * bx; fy[k] += fr2 * by; fz[k] += fr2 * bz;
  }
}

/* One torsion i-j-k-l (md_ftors.c:161-289): with a = ri - rj, b = rj - rk,
   c = rk - rl and the plane normals d = a x b, e = b x c, cos(phi) =
   d.e / (|d| |e|).  dcos/dr of atom m is (dF_m - cos dG_m) / (|d| |e|), F = d.e
   and G = |d| |e|; u1..u4 receive dU/dcos times that (the force is its
   negative).  Returns cos(phi); *pot gets U, *dudcos_out dU/dcos / G. */
typedef struct {
  double a[3], b[3], c[3];
  double dudcos;                         /* dU/dcos / G */
  double u4[3];                          /* dF_4 - cos dG_4 */
  double g1[3], g2[3], g3[3], g4[3];     /* dudcos (dF_m - cos dG_m) */
} tors_terms;

static double torsion(orc *o, int nt, double *pot, tors_terms *T)
{
  int i = o->itors[nt], j = o->jtors[nt], k = o->ktors[nt], l = o->ltors[nt];
  int t = o->idxtors[nt], row = o->tors_row[t], m;
  double ax = o->px[i] - o->px[j], ay = o->py[i] - o->py[j], az = o->pz[i] - o->pz[j];
  double bx = o->px[j] - o->px[k], by = o->py[j] - o->py[k], bz = o->pz[j] - o->pz[k];
  double cx = o->px[k] - o->px[l], cy = o->py[k] - o->py[l], cz = o->pz[k] - o->pz[l];
  double dx = ay * bz - az * by, dy = az * bx - ax * bz, dz = ax * by - ay * bx;
  double dl = sqrt(dx * dx + dy * dy + dz * dz);
  double ex = by * cz - bz * cy, ey = bz * cx - bx * cz, ez = bx * cy - by * cx;
  double el = sqrt(ex * ex + ey * ey + ez * ez);
  double cphi = (dx * ex + dy * ey + dz * ez) / (dl * el);
  double dudcos = 0., g, dre, erd;
  if (o->tors_form[t] == 0) {
    /* harmonic in phi (md_ftors.c:194-210, energy :362-381) */
    double phi = 0., dphi;
    if (cphi >= 1.0 || cphi <= -1.0) {
      dphi = phi - o->eqtors[row];
      dudcos = 0.;
    } else {
      phi = acos(cphi);
      dphi = phi - o->eqtors[row];
      dudcos = (o->fktors[row] * dphi) * (-1. / sqrt(1. - cphi * cphi));
    }
    *pot = .5 * o->fktors[row] * dphi * dphi;
  } else {
    /* power series in cos(phi) (md_ftors.c:211-220, energy :382-394) */
    const double *v = o->vphi + (size_t)row * CM3D_NB_MAXPOWER_TORS;
    double tpot = v[CM3D_NB_MAXPOWER_TORS - 1];
    dudcos = ((double)CM3D_NB_MAXPOWER_TORS - 1.) * v[CM3D_NB_MAXPOWER_TORS - 1];
    for (m = CM3D_NB_MAXPOWER_TORS - 2; m > 0; m--) dudcos = dudcos * cphi + v[m] * (double)m;
    for (m = CM3D_NB_MAXPOWER_TORS - 2; m >= 0; m--) tpot = tpot * cphi + v[m];
    *pot = tpot;
  }
  g = dl * el;
  dre = dl / el;
  erd = el / dl;
  dudcos *= 1. / g;
  T->a[0] = ax; T->a[1] = ay; T->a[2] = az;
  T->b[0] = bx; T->b[1] = by; T->b[2] = bz;
  T->c[0] = cx; T->c[1] = cy; T->c[2] = cz;
  {
    double f1x = by * ez - bz * ey, f1y = bz * ex - bx * ez, f1z = bx * ey - by * ex;
    double f2x = (cy * dz - cz * dy + (az + bz) * ey - (ay + by) * ez);
    double f2y = (cz * dx - cx * dz + (ax + bx) * ez - (az + bz) * ex);
    double f2z = (cx * dy - cy * dx + (ay + by) * ex - (ax + bx) * ey);
    double f3x = (ay * ez - az * ey + (bz + cz) * dy - (by + cy) * dz);
    double f3y = (az * ex - ax * ez + (bx + cx) * dz - (bz + cz) * dx);
    double f3z = (ax * ey - ay * ex + (by + cy) * dx - (bx + cx) * dy);
    double f4x = by * dz - bz * dy, f4y = bz * dx - bx * dz, f4z = bx * dy - by * dx;
    double h1x = (by * dz - bz * dy) * erd, h1y = (bz * dx - bx * dz) * erd, h1z = (bx * dy - by * dx) * erd;
    double h2x = ((dy * (az + bz) - dz * (ay + by)) * erd + (cy * ez - cz * ey) * dre);
    double h2y = ((dz * (ax + bx) - dx * (az + bz)) * erd + (cz * ex - cx * ez) * dre);
    double h2z = ((dx * (ay + by) - dy * (ax + bx)) * erd + (cx * ey - cy * ex) * dre);
    double h3x = ((ay * dz - az * dy) * erd + (ey * (bz + cz) - ez * (by + cy)) * dre);
    double h3y = ((az * dx - ax * dz) * erd + (ez * (bx + cx) - ex * (bz + cz)) * dre);
    double h3z = ((ax * dy - ay * dx) * erd + (ex * (by + cy) - ey * (bx + cx)) * dre);
    double h4x = (by * ez - bz * ey) * dre, h4y = (bz * ex - bx * ez) * dre, h4z = (bx * ey - by * ex) * dre;
    T->g1[0] = dudcos * (f1x - cphi * h1x); T->g1[1] = dudcos * (f1y - cphi * h1y); T->g1[2] = dudcos * (f1z - cphi * h1z);
    T->g2[0] = dudcos * (f2x - cphi * h2x); T->g2[1] = dudcos * (f2y - cphi * h2y); T->g2[2] = dudcos * (f2z - cphi * h2z);
    T->g3[0] = dudcos * (f3x - cphi * h3x); T->g3[1] = dudcos * (f3y - cphi * h3y); T->g3[2] = dudcos * (f3z - cphi * h3z);
    T->u4[0] = f4x - cphi * h4x; T->u4[1] = f4y - cphi * h4y; T->u4[2] = f4z - cphi * h4z;
    T->g4[0] = dudcos * T->u4[0]; T->g4[1] = dudcos * T->u4[1]; T->g4[2] = dudcos * T->u4[2];
    T->dudcos = dudcos;
  }
  return cphi;
}

/* ftors  energy/intra/md_ftors.c:117-293: fxr -= dU/dcos dcos/dr */
void orc_ftors(orc *o)
{
  int nt, c, n = o->n;
  for (nt = 0; nt < o->ntors; nt++) {
    int at[4] = {o->itors[nt], o->jtors[nt], o->ktors[nt], o->ltors[nt]};
    double pot;
    tors_terms T;
    torsion(o, nt, &pot, &T);
    for (c = 0; c < 3; c++) o->fxr[c * n + at[0]] -= T.g1[c];
    for (c = 0; c < 3; c++) o->fxr[c * n + at[1]] -= T.g2[c];
    for (c = 0; c < 3; c++) o->fxr[c * n + at[2]] -= T.g3[c];
    for (c = 0; c < 3; c++) o->fxr[c * n + at[3]] -= T.g4[c];
  }
}

/* quadratic interpolation of a 1-4 table at squared distance dis2
   (md_fonefour.c:124-140); *under is set (and the first knot used) below
   the table's start */
static double onfo_interp(orc *o, const double *tab, int t, double dis2, int *under)
{
  double p = (dis2 - o->r14min2[t]) * o->dx214tab[t];
  int k = (int)p;
  const double *v = tab + (size_t)t * o->n14table;
  double fm1, f0, f1;
  if (k < 1) {
    *under = 1;
    k = 1;
    p = 1.;
  }
  p = p - (double)k;
  fm1 = v[k - 1];
  f0 = v[k];
  f1 = v[k + 1];
  return f0 + .5 * p * (f1 - fm1 + p * (fm1 - 2. * f0 + f1));
}

/* fonfo  energy/intra/md_fonefour.c:70-157: tabulated 1-4 force (scaled by
   scale_onefour) plus the bare 1-4 Coulomb force (scaled by
   scale_onefour_e), within r14max */
void orc_fonfo(orc *o)
{
  int k14, n = o->n;
  double *fx = o->fxr, *fy = o->fxr + n, *fz = o->fxr + 2 * n;
  for (k14 = 0; k14 < o->n14; k14++) {
    int i = o->i14[k14], j = o->j14[k14], t = o->i14dx[k14], under = 0;
    double xd = o->px[i] - o->px[j], yd = o->py[i] - o->py[j], zd = o->pz[i] - o->pz[j];
    double dis2 = xd * xd + yd * yd + zd * zd, fcc, qij;
    if (!(dis2 < o->r14max2[t])) continue;
    fcc = onfo_interp(o, o->dv14tab, t, dis2, &under) * o->scale14;
    if (under) o->underflows++;
    if ((qij = o->qch[i] * o->qch[j]) != 0) fcc -= qij * o->scale14e / (sqrt(dis2) * dis2);
    xd *= fcc; yd *= fcc; zd *= fcc;
    fx[i] -= xd; fy[i] -= yd; fz[i] -= zd;
    fx[j] += xd; fy[j] += yd; fz[j] += zd;
  }
}

/* getvtors / getvonfo / getvbondx  md_ftors.c:296-542 (PRESSURE on, as that
   file defines it), md_fonefour.c:160-314, md_fbocross.c:100-168 */
static void tors_energies(orc *o)
{
  int nt, k14, nb, r, c;
  double st[9] = {0}, spot = 0., sprs = 0., spelec = 0., swelec = 0., sw[9] = {0}, se[9] = {0};
  o->vtors = 0.;
  for (nt = 0; nt < o->ntors; nt++) {
    double pot;
    tors_terms T;
    torsion(o, nt, &pot, &T);
    o->vtors += pot;
    /* the i-j, j-k and j-l separations times the forces on i, k and l
       (md_ftors.c:483-519) */
    for (r = 0; r < 3; r++)
      for (c = 0; c < 3; c++) st[3 * r + c] -= T.a[r] * T.g1[c];
    for (r = 0; r < 3; r++)
      for (c = 0; c < 3; c++) st[3 * r + c] += T.b[r] * T.g3[c];
    for (r = 0; r < 3; r++)
      for (c = 0; c < 3; c++) st[3 * r + c] += (T.b[r] + T.c[r]) * T.dudcos * T.u4[c];
  }
  for (c = 0; c < 9; c++) o->wtorst[c] = st[c];
  o->wtors = st[0] + st[4] + st[8];
  for (k14 = 0; k14 < o->n14; k14++) {
    int i = o->i14[k14], j = o->j14[k14], t = o->i14dx[k14], under = 0;
    double d[3] = {o->px[i] - o->px[j], o->py[i] - o->py[j], o->pz[i] - o->pz[j]};
    double dis2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2], f, qij;
    if (!(dis2 < o->r14max2[t])) continue;
    spot += onfo_interp(o, o->v14tab, t, dis2, &under);
    f = onfo_interp(o, o->dv14tab, t, dis2, &under);
    sprs -= dis2 * f;
    for (r = 0; r < 3; r++)
      for (c = 0; c < 3; c++) sw[3 * r + c] -= d[c] * d[r] * f;
    if ((qij = o->qch[i] * o->qch[j]) != 0) {
      f = qij / sqrt(dis2);
      spelec += f;
      swelec += f;
      for (r = 0; r < 3; r++)
        for (c = 0; c < 3; c++) se[3 * r + c] += f * d[c] * d[r] / dis2;
    }
  }
  o->vonfo = spot * o->scale14;
  o->wonfo = sprs * o->scale14;
  o->vonfo_e = spelec * o->scale14e;
  o->wonfo_e = swelec * o->scale14e;
  for (c = 0; c < 9; c++) {
    o->wonfot[c] = sw[c] * o->scale14;
    o->wonfoet[c] = se[c] * o->scale14e;
  }
  for (c = 0; c < 9; c++) o->wbondxt[c] = 0.;
  spot = sprs = 0.;
  for (nb = 0; nb < o->nbondx; nb++) {
    int i = o->ibondx[nb], j = o->jbondx[nb], k = o->kbondx[nb], t = o->idxbondx[nb];
    double a[3] = {o->px[i] - o->px[j], o->py[i] - o->py[j], o->pz[i] - o->pz[j]};
    double b[3] = {o->px[j] - o->px[k], o->py[j] - o->py[k], o->pz[j] - o->pz[k]};
    double al = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]), bl = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
    double dr1 = al - o->eq1bondx[t], dr2 = bl - o->eq2bondx[t], fk = o->fkbondx[t];
    spot += fk * dr1 * dr2;
    sprs -= fk * (bl * dr1 + al * dr2);
    for (r = 0; r < 3; r++)
      for (c = 0; c < 3; c++) o->wbondxt[3 * r + c] -= fk * (dr1 * b[c] * b[r] / bl + dr2 * a[c] * a[r] / al);
  }
  o->vbond += spot;
  o->wbond += sprs;
}

/* rmass  utils/md_util.new.c:219 */
void orc_rmass(orc *o, int which)
{
  double *b = block(o, which);
  int i, n = o->n;
  for (i = 0; i < n; i++) {
    double r = 1. / o->amass[i];
    b[i] *= r;
    b[i + n] *= r;
    b[i + 2 * n] *= r;
  }
}

/* freeze_atom  md_fcntr.c:311-329: frozen atoms lose their velocity and
   every force block */
static void freeze_atoms(orc *o)
{
  int f, c, n = o->n;
  for (f = 0; f < o->nfreeze; f++) {
    int j = o->ifreeze[f];
    o->vx[j] = o->vy[j] = o->vz[j] = 0.;
    for (c = 0; c < 3; c++) o->fxs[c * n + j] = o->fxl[c * n + j] = o->fxa[c * n + j] = o->fxr[c * n + j] = 0.;
  }
}

/* force  energy/control/md_fcntr.c:44-134 (levels 0-3) */
void orc_force(orc *o, int iflg)
{
  switch (iflg) {
    case 0:
      orc_zero_forces(o, 1);
      orc_force_ter(o, 0);
      orc_force_ter_e(o, 0);
      orc_rmass(o, 1);
      break;
    case 1:
      orc_zero_forces(o, 1);
      orc_zero_forces(o, 0);
      orc_force_ter(o, 1);
      orc_force_ter_e(o, 1);
      if (o->iperd == 3) {
        orc_fk_ewald(o);
        orc_ecorr(o);
      }
      orc_rmass(o, 0);
      orc_rmass(o, 1);
      break;
    case 2:
      orc_zero_forces(o, 2);
      orc_fbond(o);
      orc_fbend(o);
      orc_fbondx(o);
      orc_rmass(o, 2);
      break;
    case 3:
      orc_zero_forces(o, 3);
      orc_ftors(o);
      orc_fonfo(o);
      orc_rmass(o, 3);
      break;
    default:
      return;
  }
  freeze_atoms(o);
}

/* getvbond / getvbend energies and virials  md_fbond.c:131-220,
   md_fbend.c:262-410.  md_fbend.c:38 defines PRESSURE for its own file, so the
   bend virial is always on: a scalar that vanishes up to rounding (an angle
   does not change under a uniform dilation) and a traceless tensor, formed
   from the atoms' absolute positions */
static void bonded_energies(orc *o)
{
  int nb, i;
  o->vbond = o->wbond = o->vbend = o->wbend = 0.;
  for (i = 0; i < 9; i++) o->wbondt[i] = o->wbendt[i] = 0.;
  for (nb = 0; nb < o->nbonds; nb++) {
    int a = o->ibond[nb], b = o->jbond[nb], idx = o->idxbond[nb];
    double dx = o->px[a] - o->px[b], dy = o->py[a] - o->py[b], dz = o->pz[a] - o->pz[b];
    double r = sqrt(dx * dx + dy * dy + dz * dz), dr = r - o->eqbond[idx];
    double fk = o->fkbond[idx];
    o->vbond += .5 * fk * dr * dr;
    fk = fk * dr / r;
    o->wbond -= fk * r * r;
    o->wbondt[0] -= fk * dx * dx; o->wbondt[1] -= fk * dy * dx; o->wbondt[2] -= fk * dz * dx;
    o->wbondt[3] -= fk * dx * dy; o->wbondt[4] -= fk * dy * dy; o->wbondt[5] -= fk * dz * dy;
    o->wbondt[6] -= fk * dx * dz; o->wbondt[7] -= fk * dy * dz; o->wbondt[8] -= fk * dz * dz;
  }
  for (nb = 0; nb < o->nbends; nb++) {
    int a = o->ibend[nb], b = o->jbend[nb], c = o->kbend[nb], idx = o->idxbend[nb];
    double ax = o->px[a] - o->px[b], ay = o->py[a] - o->py[b], az = o->pz[a] - o->pz[b];
    double al = ax * ax + ay * ay + az * az;
    double bx = o->px[c] - o->px[b], by = o->py[c] - o->py[b], bz = o->pz[c] - o->pz[b];
    double bl = bx * bx + by * by + bz * bz;
    double r11 = 1. / sqrt(al * bl), costh = (ax * bx + ay * by + az * bz) * r11, th, dth;
    costh = costh < 1. ? costh : 1.;
    costh = costh > -1. ? costh : -1.;
    th = fabs(costh) >= 1. ? 1. : acos(costh);
    dth = th - o->eqbend[idx];
    o->vbend += .5 * o->fkbend[idx] * dth * dth;
    {
      /* harmonic: dU/dth = 0 at |cos| = 1 (md_fbend.c:322-327) */
      double dudth = fabs(costh) >= 1. ? 0. : o->fkbend[idx] * dth;
      double dthdcos = fabs(costh) >= 1. ? -1. : -1. / sqrt(1. - costh * costh);
      double dudcos = dudth * dthdcos;
      double c1x = costh * ax / al - bx * r11, c1y = costh * ay / al - by * r11, c1z = costh * az / al - bz * r11;
      double c2x = -costh * (ax / al + bx / bl) + (ax + bx) * r11;
      double c2y = -costh * (ay / al + by / bl) + (ay + by) * r11;
      double c2z = -costh * (az / al + bz / bl) + (az + bz) * r11;
      double c3x = costh * bx / bl - ax * r11, c3y = costh * by / bl - ay * r11, c3z = costh * bz / bl - az * r11;
      double xi = o->px[a], xj = o->px[b], xk = o->px[c];
      double yi = o->py[a], yj = o->py[b], yk = o->py[c];
      double zi = o->pz[a], zj = o->pz[b], zk = o->pz[c];
      o->wbend += dudcos * (ax * c1x + ay * c1y + az * c1z - bx * c3x - by * c3y - bz * c3z);
      o->wbendt[0] += dudcos * (xi * c1x + xj * c2x + xk * c3x);
      o->wbendt[1] += dudcos * (yi * c1x + yj * c2x + yk * c3x);
      o->wbendt[2] += dudcos * (zi * c1x + zj * c2x + zk * c3x);
      o->wbendt[3] += dudcos * (xi * c1y + xj * c2y + xk * c3y);
      o->wbendt[4] += dudcos * (yi * c1y + yj * c2y + yk * c3y);
      o->wbendt[5] += dudcos * (zi * c1y + zj * c2y + zk * c3y);
      o->wbendt[6] += dudcos * (xi * c1z + xj * c2z + xk * c3z);
      o->wbendt[7] += dudcos * (yi * c1z + yj * c2z + yk * c3z);
      o->wbendt[8] += dudcos * (zi * c1z + zj * c2z + zk * c3z);
    }
  }
}

/* getvireal(...,1) + geteng  md_fcntr.c:136-308 for the terms of this path */
void orc_get_energies(orc *o, cm3d_nb_energies *e)
{
  int i, n = o->n;
  double vol = get_deth(o->hmat), rvol = 1. / vol, p2m;
  memset(e, 0, sizeof *e);
  e->vhinter = o->spothl;
  e->vinter = o->spotl;
  e->winter = o->sprsl;
  for (i = 0; i < 9; i++) e->wintertensor[i] = o->sprslt[i];
  e->velec = o->spote;
  e->welec = o->sprse;
  for (i = 0; i < 9; i++) e->welectensor[i] = o->sprset[i];
  if (o->iperd == 3) {
    e->vewald = o->vk_ewald + o->pot_ecorr;
    e->wewald = o->vp_ewald + o->prs_ecorr;
    for (i = 0; i < 9; i++) e->wewaldtensor[i] = o->vp_ewald_tensor[i] + o->prs_ecorr_tensor[i];
  }
  bonded_energies(o);
  tors_energies(o);
  e->vbond = o->vbond;
  e->wbond = o->wbond;
  e->vbend = o->vbend;
  e->wbend = o->wbend;
  e->US = e->vhinter + e->velec + e->vewald;
  e->U = e->vinter + e->velec + e->vewald;
  e->W = e->winter + e->welec + e->wewald;
  for (i = 0; i < 9; i++) e->Wtensor[i] = e->wintertensor[i] + e->welectensor[i] + e->wewaldtensor[i];
  if (o->iperd == 3) {
    e->W -= 3 * o->wlrc * rvol;
    e->Wtensor[0] -= o->wlrc * rvol;
    e->Wtensor[4] -= o->wlrc * rvol;
    e->Wtensor[8] -= o->wlrc * rvol;
  }
  /* get_p2mt  md_fcntr.c:332-354 */
  for (i = 0; i < n; i++) {
    double am = o->amass[i];
    e->p2m_tensor[0] += am * (o->vx[i] * o->vx[i]);
    e->p2m_tensor[4] += am * (o->vy[i] * o->vy[i]);
    e->p2m_tensor[8] += am * (o->vz[i] * o->vz[i]);
    e->p2m_tensor[1] += am * (o->vy[i] * o->vx[i]);
    e->p2m_tensor[2] += am * (o->vz[i] * o->vx[i]);
    e->p2m_tensor[5] += am * (o->vz[i] * o->vy[i]);
  }
  e->p2m_tensor[3] = e->p2m_tensor[1];
  e->p2m_tensor[6] = e->p2m_tensor[2];
  e->p2m_tensor[7] = e->p2m_tensor[5];
  p2m = e->p2m_tensor[0] + e->p2m_tensor[4] + e->p2m_tensor[8];
  {
    /* UI, WI and WItensor as getvireal sums them (md_fcntr.c:205-215) */
    double UI, WI, *wit = e->WItensor;
    e->vtors = o->vtors;
    e->wtors = o->wtors;
    e->vonfo = o->vonfo;
    e->vonfo_e = o->vonfo_e;
    e->wonfo = o->wonfo;
    e->wonfo_e = o->wonfo_e;
    UI = e->vbond + e->vbend + e->vtors + e->vonfo + e->vonfo_e;
    WI = e->wbond + e->wbend + e->wtors + e->wonfo + e->wonfo_e;
    for (i = 0; i < 9; i++)
      wit[i] = o->wbondt[i] + o->wbendt[i] + o->wtorst[i] + o->wonfot[i] + o->wonfoet[i] + o->wbondxt[i];
    e->UI = UI;
    e->WI = WI;
    e->poth = e->US;
    e->poter = e->U;
    e->potra = UI;
    if (o->iperd == 3) {
      e->poter += o->vlrc / vol;
      e->poth += o->vlrc / vol;
    }
    e->prsi = (p2m + e->W + WI) / (3 * vol);
    for (i = 0; i < 9; i++) e->prs_tensor[i] = (e->p2m_tensor[i] + e->Wtensor[i] + wit[i]) / vol;
  }
  e->zke = .5 * p2m;
  e->tiout = p2m / (double)o->ndof;
}

/* Nose-Hoover chains.  forcen_new (integrate/md_therm.new.c:175-198): the
   thermostats' kinetic sums and the chain forces.  An atom without a
   thermostat (ithm -1) adds to no sum here; CM3D would write p2mt[-1]. */
static void nhc_forces(orc *o)
{
  int i, j, n = o->n, nc = o->nchain;
  for (j = 0; j < o->ntherm; j++) o->p2mt[j] = 0.;
  for (i = 0; i < n; i++)
    if (o->ithm[i] >= 0)
      o->p2mt[o->ithm[i]] += o->amass[i] * (o->vx[i] * o->vx[i] + o->vy[i] * o->vy[i] + o->vz[i] * o->vz[i]);
  for (j = 0; j < o->ntherm; j++) {
    double *f = o->feta + (size_t)j * nc, *m = o->mnh + (size_t)j * nc, *g = o->gkt + (size_t)j * nc,
           *v = o->veta + (size_t)j * nc;
    f[0] = (o->p2mt[j] - g[0]) / m[0];
    for (i = 1; i < nc; i++) f[i] = (m[i - 1] * v[i - 1] * v[i - 1] - g[i]) / m[i];
  }
}

/* the atoms' velocity scaling by exp(-dt/2 veta_0) of their thermostat */
static void nhc_scale(orc *o, double dta2)
{
  int i, n = o->n;
  for (i = 0; i < n; i++) {
    double e = o->ithm[i] >= 0 ? exp(-dta2 * o->veta[(size_t)o->ithm[i] * o->nchain]) : exp(-dta2 * 0.);
    o->vx[i] *= e;
    o->vy[i] *= e;
    o->vz[i] *= e;
  }
}

/* intnhc_new  integrate/md_therm.new.c:278-333: one thermostat half step of
   dta2 in CM3D's order (scale, chain links from the top, forces, chain
   velocities and positions, links from the bottom, scale) */
static void intnhc(orc *o, double dta2)
{
  int i, j, nc = o->nchain, nt = o->ntherm;
  double dta = 2. * dta2;
  double *v = o->veta, *f = o->feta, *m = o->mnh, *g = o->gkt;
  nhc_scale(o, dta2);
  for (i = 0; i < nc - 1; i++)
    for (j = 0; j < nt; j++) v[(size_t)j * nc + i] *= exp(-dta2 * v[(size_t)j * nc + i + 1]);
  nhc_forces(o);
  for (i = 0; i < nc; i++)
    for (j = 0; j < nt; j++) v[(size_t)j * nc + i] += dta2 * f[(size_t)j * nc + i];
  for (i = 0; i < nc; i++)
    for (j = 0; j < nt; j++) o->eta[(size_t)j * nc + i] += dta * v[(size_t)j * nc + i];
  for (j = 0; j < nt; j++) v[(size_t)j * nc] += dta2 * f[(size_t)j * nc];
  for (i = 1; i < nc; i++)
    for (j = 0; j < nt; j++) {
      size_t k = (size_t)j * nc + i;
      v[k] += dta2 * (m[k - 1] * v[k - 1] * v[k - 1] - g[k]) / m[k];
    }
  for (i = nc - 2; i >= 0; i--)
    for (j = 0; j < nt; j++) v[(size_t)j * nc + i] *= exp(-dta2 * v[(size_t)j * nc + i + 1]);
  nhc_scale(o, dta2);
}

void orc_get_nhc(orc *o, double *eta, double *veta)
{
  size_t tc = (size_t)o->ntherm * o->nchain;
  if (tc) {
    memcpy(eta, o->eta, tc * 8);
    memcpy(veta, o->veta, tc * 8);
  }
}

/* nrefsh  energy/control/md_finter.c:43-108 (verlist branch) */
static void nrefsh(orc *o, int istep)
{
  int i, n = o->n, iflag = 0;
  double skin2 = .25 * o->skin * o->skin;
  for (i = 0; i < n; i++) {
    double xc = o->dxn[i] - o->px[i], yc = o->dxn[i + n] - o->py[i], zc = o->dxn[i + 2 * n] - o->pz[i];
    if (xc * xc + yc * yc + zc * zc > skin2) {
      iflag = 1;
      break;
    }
  }
  if (iflag) {
    if (istep - o->isteplast < 3) {
      o->resets++;
      for (i = 0; i < n; i++) {
        double xc = o->px[i] - o->dxn[i], yc = o->py[i] - o->dxn[i + n], zc = o->pz[i] - o->dxn[i + 2 * n];
        if (xc * xc + yc * yc + zc * zc > skin2) {
          double scale = skin2 / (xc * xc + yc * yc + zc * zc);
          o->px[i] = o->dxn[i] + scale * xc;
          o->py[i] = o->dxn[i + n] + scale * yc;
          o->pz[i] = o->dxn[i + 2 * n] + scale * zc;
        }
      }
    }
    orc_get_ngbr(o);
    o->isteplast = istep;
  }
}

/* step_init  integrate/md_step.c:32-59 (nonbonded + bonded levels) */
void orc_step_init(orc *o)
{
  o->isteplast = 0;
  orc_get_ngbr(o);
  orc_force(o, 1);
  orc_force(o, 2);
  orc_force(o, 3);
}

/* step  integrate/md_step.c:62-159 (NVE, or NVT with Nose-Hoover chains) */
void orc_step(orc *o, int istep0, int nsteps)
{
  int s, n3 = 3 * o->n, i;
  int ninter = o->nres_lrf, ninrra = o->nres_tors, ninnra = o->nres_intra;
  double dtl2 = .5 * o->dt, dts2 = dtl2 / (double)ninter, dtr2 = dts2 / (double)ninrra;
  double dta2 = dtr2 / (double)ninnra, dter = (double)ninter * dts2,
         dter1 = (double)(1 - ninter) * dts2;
  double *pos = o->px, *vel = o->vx;
  /* CM3D keeps px,py,pz (and vx,vy,vz) contiguous (md_util.new.c:113-119) and
     loops over 3N; the oracle keeps separate arrays, so loop per block */
  double *P[3] = {o->px, o->py, o->pz}, *V[3] = {o->vx, o->vy, o->vz};
  int n = o->n;
  (void)pos; (void)vel; (void)n3;
  for (s = 0; s < nsteps; s++) {
    int istep = istep0 + s, intr, inrra, intra, c;
    for (intr = 0; intr < ninter; intr++) {
      for (c = 0; c < 3; c++) {
        if (intr == 0) {
          for (i = 0; i < n; i++) V[c][i] += dter * o->fxl[c * n + i] + dter1 * o->fxs[c * n + i];
        } else {
          for (i = 0; i < n; i++) V[c][i] += dts2 * o->fxs[c * n + i];
        }
      }
      for (inrra = 0; inrra < ninrra; inrra++) {
        for (c = 0; c < 3; c++)
          for (i = 0; i < n; i++) V[c][i] += dtr2 * o->fxr[c * n + i];
        for (intra = 0; intra < ninnra; intra++) {
          for (c = 0; c < 3; c++)
            for (i = 0; i < n; i++) V[c][i] += dta2 * o->fxa[c * n + i];
          for (c = 0; c < 3; c++)
            for (i = 0; i < n; i++) P[c][i] += dta2 * V[c][i];
          if (o->ntherm) intnhc(o, dta2);    /* md_step.c:117 (no barostat) */
          for (c = 0; c < 3; c++)
            for (i = 0; i < n; i++) P[c][i] += dta2 * V[c][i];
          orc_force(o, 2);
          for (c = 0; c < 3; c++)
            for (i = 0; i < n; i++) V[c][i] += dta2 * o->fxa[c * n + i];
        }
        orc_force(o, 3);
        for (c = 0; c < 3; c++)
          for (i = 0; i < n; i++) V[c][i] += dtr2 * o->fxr[c * n + i];
      }
      nrefsh(o, istep);
      if (intr == ninter - 1) {
        orc_force(o, 1);
        for (c = 0; c < 3; c++)
          for (i = 0; i < n; i++) V[c][i] += dter * o->fxl[c * n + i] + dter1 * o->fxs[c * n + i];
      } else {
        orc_force(o, 0);
        for (c = 0; c < 3; c++)
          for (i = 0; i < n; i++) V[c][i] += dts2 * o->fxs[c * n + i];
      }
    }
  }
}

long long orc_rebuilds(orc *o) { return o->rebuilds; }
long long orc_resets(orc *o) { return o->resets; }
long long orc_underflows(orc *o) { return o->underflows; }
