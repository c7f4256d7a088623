/*
 * ref_dump.c -- full-precision dump harness for the CM3D reference.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is compiled against the reference's
 * own headers and linked against the reference's own archives (see
 * oracle/Makefile); it is never part of the product.
 *
 * It replays the start of CM3D's MD driver
 *   main_new            main/md_main.new.c:61-101
 *   md_mdcntr_new       main/md_mdcntr.new.c:87-127  (readpos, samvel, step_init)
 * and then writes every quantity on the nonbonded hot path at full precision
 * (raw IEEE doubles / int32), because CM3D's own writers print forces with
 * %g (output/md_saveout.c:65), far too coarse for parity checks.
 *
 * usage:  ref_dump <cm3d input file> <out.bin> [nsteps]
 *   run from the directory holding the input (CM3D opens files relative to
 *   the current directory).
 *
 * File format: "CM3DDUMP" then records of
 *   char name[32]; int32 kind (1=f64, 2=i32); int64 count; payload.
 */
#include "md.h"

static FILE *g_out;

static void rec(const char *name, int kind, long long n, const void *data)
{
  char nm[32];
  int k = kind;
  memset(nm, 0, sizeof nm);
  strncpy(nm, name, 31);
  fwrite(nm, 1, 32, g_out);
  fwrite(&k, sizeof k, 1, g_out);
  fwrite(&n, sizeof n, 1, g_out);
  if (n > 0) fwrite(data, kind == 1 ? 8 : 4, (size_t)n, g_out);
}
static void recd(const char *name, long long n, const double *d) { rec(name, 1, n, d); }
static void reci(const char *name, long long n, const int *d) { rec(name, 2, n, d); }
static void rec1d(const char *name, double v) { recd(name, 1, &v); }
static void rec1i(const char *name, int v) { reci(name, 1, &v); }

/* forces are stored by CM3D as accelerations (md_fcntr.c:74-75); convert a
   triple of SoA blocks back to forces before writing */
static void rec_force(const char *name, int n, const double *fx, const double *fy,
                      const double *fz, const double *amass, int is_accel)
{
  double *buf = (double *)malloc(3 * (size_t)n * sizeof(double));
  int i;
  for (i = 0; i < n; i++) {
    double m = is_accel ? amass[i] : 1.0;
    buf[i] = fx[i] * m;
    buf[n + i] = fy[i] * m;
    buf[2 * n + i] = fz[i] * m;
  }
  recd(name, 3LL * n, buf);
  free(buf);
}

static void zero3(double *a, double *b, double *c, int n)
{
  int i;
  for (i = 0; i < n; i++) a[i] = b[i] = c[i] = 0.0;
}

static void dump_energies(const char *pfx, ENERGIES *e)
{
  char nm[64];
#define E1(f) do { snprintf(nm, sizeof nm, "%s" #f, pfx); rec1d(nm, e->f); } while (0)
#define E9(f) do { snprintf(nm, sizeof nm, "%s" #f, pfx); recd(nm, 9, e->f); } while (0)
  E1(vinter); E1(vhinter); E1(velec); E1(vewald); E1(vbond); E1(vbend);
  E1(winter); E1(welec); E1(wewald); E1(wbond); E1(wbend);
  E1(US); E1(U); E1(W); E1(UI); E1(WI);
  E9(wintertensor); E9(welectensor); E9(wewaldtensor); E9(Wtensor);
  E1(prsi); E9(prs_tensor); E1(zke); E1(tiout); E1(poth); E1(poter); E1(potra);
  E1(vtors); E1(vonfo); E1(vonfo_e); E1(vbondx); E1(wtors); E1(wonfo); E1(wonfo_e); E1(wbondx);
  E9(wtorstensor); E9(wonfotensor); E9(wonfo_etensor); E9(wbondxtensor); E9(WItensor);
#undef E1
#undef E9
}

int main(int argc, char *argv[])
{
  SIMPARMS simparms;
  FILENAMES filenames;
  COORDS coords;
  SUBSPACE subspace;
  WRITE_STEP write_step;
  NGBR ngbr;
  INTER inter;
  ENERGIES energies;
  int i, n, nsteps = 0, ninter, ntable;
  double *save;

  if (argc < 3) {
    fprintf(stderr, "usage: %s input out.bin [nsteps]\n", argv[0]);
    return 2;
  }
  if (argc > 3) nsteps = atoi(argv[3]);

  memset(&simparms, 0, sizeof simparms);
  memset(&filenames, 0, sizeof filenames);
  memset(&coords, 0, sizeof coords);
  memset(&subspace, 0, sizeof subspace);
  memset(&write_step, 0, sizeof write_step);
  memset(&ngbr, 0, sizeof ngbr);
  memset(&inter, 0, sizeof inter);
  memset(&energies, 0, sizeof energies);
  simparms.mem_bytes = 0;
  simparms.rank = 0;
  simparms.size = 1;
  strcpy(filenames.infile, argv[1]);
  strcpy(filenames.command, argv[0]);

  md_startup(&filenames, &simparms, &subspace, &write_step, &inter, &ngbr, &coords);
  if (simparms.icalc_type != 0) {
    fprintf(stderr, "ref_dump: only calculation{md} inputs are supported\n");
    return 2;
  }

  readpos(argv[0], filenames.initfile, &simparms, &energies.estep, &energies, &coords);
  if (simparms.istart == 1) {
    samvel(&simparms, &coords, 1);
    samveta(&simparms, &coords);
    if (simparms.ivol) samvbar(&simparms, &coords);
  }
  zero_averages(&simparms, &energies);
  gethinv9(coords.hmat, coords.hmati);
  step_init(&simparms, &coords, &energies, &inter, &ngbr);

  n = simparms.natoms;
  ninter = inter.ntype;
  ntable = inter.ntable;

  g_out = fopen(argv[2], "wb");
  if (!g_out) { perror(argv[2]); return 1; }
  fwrite("CM3DDUMP", 1, 8, g_out);

  /* ---- system description (the engine's inputs) ---- */
  rec1i("natoms", n);
  rec1i("iperd", simparms.iperd);
  rec1i("ivol", simparms.ivol);
  rec1i("nlen", simparms.nlen);
  rec1i("nres_lrf", simparms.ninter);
  rec1i("nres_intra", simparms.ninnra);
  rec1i("nres_tors", simparms.ninrra);
  rec1i("ndof", simparms.ndof);
  rec1i("istep", simparms.istep);
  rec1d("dt", simparms.dt);
  rec1d("temp", simparms.temp);
  rec1d("vlrc", simparms.vlrc);
  rec1d("wlrc", simparms.wlrc);
  rec1i("ncells", ngbr.ncells);
  rec1i("nocell_all", simparms.nocell_all);
  rec1i("ilist", ngbr.ilist);
  recd("hmat", 9, coords.hmat);
  recd("hmati", 9, coords.hmati);
  recd("px", n, coords.px); recd("py", n, coords.py); recd("pz", n, coords.pz);
  recd("vx", n, coords.vx); recd("vy", n, coords.vy); recd("vz", n, coords.vz);
  recd("amass", n, coords.amass);
  recd("qch", n, coords.qch);
  reci("itype", n, inter.itype);
  rec1i("ntypes", simparms.ntypes);
  {
    int nt = simparms.ntypes, a, b;
    int *m = (int *)malloc(sizeof(int) * (size_t)(nt * nt > 0 ? nt * nt : 1));
    for (a = 0; a < nt; a++)
      for (b = 0; b < nt; b++) m[a * nt + b] = inter.map[a][b];
    reci("map", (long long)nt * nt, m);
    free(m);
  }
  rec1i("ninter", ninter);
  rec1i("ntable", ntable);
  recd("rmaxs_cut2", ninter, inter.rmaxs_cut2);
  recd("rmins_cut2", ninter, inter.rmins_cut2);
  recd("rmaxl_cut2", ninter, inter.rmaxl_cut2);
  recd("rminl_cut2", ninter, inter.rminl_cut2);
  recd("rmaxs_skin2", ninter, inter.rmaxs_skin2);
  recd("rmaxl_skin2", ninter, inter.rmaxl_skin2);
  recd("rminl_skin2", ninter, inter.rminl_skin2);
  recd("dx2tab", ninter, inter.dx2tab);
  recd("vtab", (long long)ninter * ntable, inter.vtab[0]);
  recd("dvtab", (long long)ninter * ntable, inter.dvtab[0]);
  recd("switchs", (long long)ninter * ntable, inter.switchs[0]);
  rec1d("skin", inter.skin_ter);
  rec1d("rheal", inter.rheal);
  rec1i("ncharge", coords.coul.ncharge);
  if (coords.coul.ncharge > 0) {
    reci("icharge", coords.coul.ncharge, coords.coul.icharge);
    recd("coultab", ntable, inter.coultab);
    recd("dcoultab", ntable, inter.dcoultab);
    recd("switchse", ntable, inter.switchse);
  }
  rec1d("dx2coul", inter.dx2coul);
  rec1d("rmins_coul2", inter.rmins_coul2);
  rec1d("rmaxs_coul2", inter.rmaxs_coul2);
  rec1d("rminl_coul2", inter.rminl_coul2);
  rec1d("rmaxl_coul2", inter.rmaxl_coul2);
  rec1d("rmaxs_skin2_e", inter.rmaxs_skin2_e);
  rec1d("rmaxl_skin2_e", inter.rmaxl_skin2_e);
  rec1d("rminl_skin2_e", inter.rminl_skin2_e);
  /* exclusions, flattened CSR (per-atom sorted lists, stored at the lower
     index of each unordered pair) */
  {
    int tot = 0, k, *off = (int *)malloc(sizeof(int) * (n + 1)), *idx;
    for (i = 0; i < n; i++) tot += inter.nexclude[i];
    idx = (int *)malloc(sizeof(int) * (tot > 0 ? tot : 1));
    off[0] = 0;
    for (i = 0; i < n; i++) {
      for (k = 0; k < inter.nexclude[i]; k++) idx[off[i] + k] = inter.exclude[i][k];
      off[i + 1] = off[i] + inter.nexclude[i];
    }
    reci("excl_off", n + 1, off);
    reci("excl_idx", tot, idx);
    free(idx);
    tot = 0;
    for (i = 0; i < n; i++) tot += coords.coul.nexclude ? coords.coul.nexclude[i] : 0;
    idx = (int *)malloc(sizeof(int) * (tot > 0 ? tot : 1));
    off[0] = 0;
    for (i = 0; i < n; i++) {
      int ne = coords.coul.nexclude ? coords.coul.nexclude[i] : 0;
      for (k = 0; k < ne; k++) idx[off[i] + k] = coords.coul.exclude[i][k];
      off[i + 1] = off[i] + ne;
    }
    reci("cexcl_off", n + 1, off);
    reci("cexcl_idx", tot, idx);
    free(idx);
    free(off);
  }
  rec1i("necorr", coords.coul.necorr);
  if (coords.coul.necorr > 0) {
    reci("iecorr", coords.coul.necorr, coords.coul.iecorr);
    reci("jecorr", coords.coul.necorr, coords.coul.jecorr);
  }
  rec1i("ktot", coords.coul.ktot);
  if (coords.coul.ktot > 0) {
    reci("ka", coords.coul.ktot, coords.coul.ka);
    reci("kb", coords.coul.ktot, coords.coul.kb);
    reci("kc", coords.coul.ktot, coords.coul.kc);
    reci("kup", coords.coul.ktot + 1, coords.coul.kup);
  }
  rec1d("kappa", coords.coul.kappa);
  rec1d("kappa2", coords.coul.kappa2);
  rec1d("falp2", coords.coul.falp2);
  rec1d("ewald_self", coords.coul.ewald_self);
  rec1d("ewald_bkg", coords.coul.ewald_bkg);
  /* harmonic bonds / bends (the inner RESPA level) */
  rec1i("nbonds", coords.bonds.nbonds);
  if (coords.bonds.nbonds > 0) {
    reci("ibond", coords.bonds.nbonds, coords.bonds.ibond);
    reci("jbond", coords.bonds.nbonds, coords.bonds.jbond);
    reci("idxbond", coords.bonds.nbonds, coords.bonds.idxbond);
    reci("itypbond", coords.bonds.itypes, coords.bonds.itypbond);
    recd("eqbond", coords.bonds.itypes, coords.bonds.eqbond);
    recd("fkbond", coords.bonds.itypes, coords.bonds.fkbond);
  }
  rec1i("nbends", coords.bends.nbends);
  if (coords.bends.nbends > 0) {
    reci("ibend", coords.bends.nbends, coords.bends.ibend);
    reci("jbend", coords.bends.nbends, coords.bends.jbend);
    reci("kbend", coords.bends.nbends, coords.bends.kbend);
    reci("idxbend", coords.bends.nbends, coords.bends.idxbend);
    reci("itypbend", coords.bends.itypes, coords.bends.itypbend);
    recd("eqbend", coords.bends.itypes, coords.bends.eqbend);
    recd("fkbend", coords.bends.itypes, coords.bends.fkbend);
  }
  /* Nose-Hoover chain thermostats (set_therm_new md_therm.new.c:32, state
     after samveta): per thermostat and chain link the masses mnh, targets
     gkt, positions eta and velocities veta; ithm maps atoms to thermostats */
  rec1i("iensemble", simparms.iensemble);
  rec1i("ntherm", simparms.ntherm);
  rec1i("nchain", simparms.nchain);
  if (simparms.ntherm > 0) {
    int t;
    double *buf = (double *)malloc(sizeof(double) * 4 * (size_t)simparms.ntherm * simparms.nchain);
    reci("ithm", n, coords.ithm);
    for (t = 0; t < simparms.ntherm; t++) {
      size_t o = (size_t)t * simparms.nchain, tot = (size_t)simparms.ntherm * simparms.nchain;
      memcpy(buf + o, coords.mnh[t], sizeof(double) * simparms.nchain);
      memcpy(buf + tot + o, coords.gkt[t], sizeof(double) * simparms.nchain);
      memcpy(buf + 2 * tot + o, coords.eta[t], sizeof(double) * simparms.nchain);
      memcpy(buf + 3 * tot + o, coords.veta[t], sizeof(double) * simparms.nchain);
    }
    recd("mnh", (long long)simparms.ntherm * simparms.nchain, buf);
    recd("gkt", (long long)simparms.ntherm * simparms.nchain, buf + (size_t)simparms.ntherm * simparms.nchain);
    recd("nhc_eta", (long long)simparms.ntherm * simparms.nchain, buf + 2 * (size_t)simparms.ntherm * simparms.nchain);
    recd("nhc_veta", (long long)simparms.ntherm * simparms.nchain, buf + 3 * (size_t)simparms.ntherm * simparms.nchain);
    free(buf);
  }
  /* frozen atoms (freeze_atom md_fcntr.c:311, applied at the end of every force level) */
  rec1i("nfreeze", simparms.nfreeze);
  if (simparms.nfreeze > 0) reci("ifreeze", simparms.nfreeze, coords.ifreeze);
  rec1i("ntors", coords.tors.ntorss);
  rec1i("n14", coords.onfo.n14s);
  rec1i("nbondx", coords.bondxs.nbondxs);
  /* torsions (the torsion RESPA level, md_ftors.c:117): per torsion its four
     atoms and type; per type the potential form (0 harmonic, 1 cosine power
     series) and the index into eqtors/fktors or vphi */
  if (coords.tors.ntorss > 0) {
    int t, nh = 0, nv = 0;
    reci("itors", coords.tors.ntorss, coords.tors.itors);
    reci("jtors", coords.tors.ntorss, coords.tors.jtors);
    reci("ktors", coords.tors.ntorss, coords.tors.ktors);
    reci("ltors", coords.tors.ntorss, coords.tors.ltors);
    reci("idxtors", coords.tors.ntorss, coords.tors.idxtors);
    reci("tors_ind_pot", coords.tors.itypes, coords.tors.ind_pot);
    reci("tors_ind_pot_num", coords.tors.itypes, coords.tors.ind_pot_num);
    for (t = 0; t < coords.tors.itypes; t++) {
      int k = coords.tors.ind_pot_num[t] + 1;
      if (coords.tors.ind_pot[t] == 0 && k > nh) nh = k;
      if (coords.tors.ind_pot[t] == 1 && k > nv) nv = k;
    }
    if (nh > 0) {
      recd("eqtors", nh, coords.tors.eqtors);
      recd("fktors", nh, coords.tors.fktors);
    }
    if (nv > 0) recd("vphi", (long long)nv * MAXPOWER_TORS, &coords.tors.vphi[0][0]);
  }
  /* 1-4 pairs (md_fonefour.c:70): tabulated potential and force per type */
  if (coords.onfo.n14s > 0) {
    int t;
    reci("i14", coords.onfo.n14s, coords.onfo.i14);
    reci("j14", coords.onfo.n14s, coords.onfo.j14);
    reci("i14dx", coords.onfo.n14s, coords.onfo.i14dx);
    rec1i("n14table", coords.onfo.n14table);
    rec1i("n14types", coords.onfo.itypes);
    recd("r14min2", coords.onfo.itypes, coords.onfo.r14min2);
    recd("r14max2", coords.onfo.itypes, coords.onfo.r14max2);
    recd("dx214tab", coords.onfo.itypes, coords.onfo.dx214tab);
    rec1d("scale_onefour", coords.onfo.scale_onefour);
    rec1d("scale_onefour_e", coords.onfo.scale_onefour_e);
    {
      double *v = (double *)malloc(sizeof(double) * 2 * (size_t)coords.onfo.itypes * coords.onfo.n14table);
      double *dv = v + (size_t)coords.onfo.itypes * coords.onfo.n14table;
      for (t = 0; t < coords.onfo.itypes; t++) {
        memcpy(v + (size_t)t * coords.onfo.n14table, coords.onfo.v14tab[t], sizeof(double) * coords.onfo.n14table);
        memcpy(dv + (size_t)t * coords.onfo.n14table, coords.onfo.dv14tab[t], sizeof(double) * coords.onfo.n14table);
      }
      recd("v14tab", (long long)coords.onfo.itypes * coords.onfo.n14table, v);
      recd("dv14tab", (long long)coords.onfo.itypes * coords.onfo.n14table, dv);
      free(v);
    }
  }
  /* cross bonds (md_fbocross.c:40) */
  if (coords.bondxs.nbondxs > 0) {
    reci("ibondx", coords.bondxs.nbondxs, coords.bondxs.ibondx);
    reci("jbondx", coords.bondxs.nbondxs, coords.bondxs.jbondx);
    reci("kbondx", coords.bondxs.nbondxs, coords.bondxs.kbondx);
    reci("idxbondx", coords.bondxs.nbondxs, coords.bondxs.idxbox);
    recd("eq1bondx", coords.bondxs.itypes, coords.bondxs.eq1bondx);
    recd("eq2bondx", coords.bondxs.itypes, coords.bondxs.eq2bondx);
    recd("fkbondx", coords.bondxs.itypes, coords.bondxs.fkbondx);
  }

  /* ---- neighbour lists after step_init (get_ngbr ngbr_list.c:297) ---- */
  rec1i("nprt", ngbr.nprt); rec1i("nprs", ngbr.nprs);
  rec1i("nprte", ngbr.nprte); rec1i("nprse", ngbr.nprse);
  if (ngbr.ilist == 1) {
    reci("inpt", ngbr.nprt, ngbr.inpt); reci("jnpt", ngbr.nprt, ngbr.jnpt);
    reci("inps", ngbr.nprs, ngbr.inps); reci("jnps", ngbr.nprs, ngbr.jnps);
    if (coords.coul.ncharge > 0) {
      reci("inpte", ngbr.nprte, ngbr.inpte); reci("jnpte", ngbr.nprte, ngbr.jnpte);
      reci("inpse", ngbr.nprse, ngbr.inpse); reci("jnpse", ngbr.nprse, ngbr.jnpse);
    }
  }

  /* ---- t=0 forces and energies from step_init ---- */
  rec_force("acc_l", n, coords.fxl, coords.fyl, coords.fzl, coords.amass, 0);
  rec_force("acc_s", n, coords.fxs, coords.fys, coords.fzs, coords.amass, 0);
  rec_force("acc_a", n, coords.fxa, coords.fya, coords.fza, coords.amass, 0);
  rec_force("acc_r", n, coords.fxr, coords.fyr, coords.fzr, coords.amass, 0);
  dump_energies("e0_", &energies);
  rec1d("vk_ewald", coords.coul.vk_ewald);
  rec1d("vp_ewald", coords.coul.vp_ewald);
  recd("vp_ewald_tensor", 9, coords.coul.vp_ewald_tensor);
  rec1d("pot_ecorr", coords.coul.pot_ecorr);
  rec1d("prs_ecorr", coords.coul.prs_ecorr);
  recd("prs_ecorr_tensor", 9, coords.coul.prs_ecorr_tensor);

  /* ---- per-term decomposition (each call into a zeroed force block) ---- */
  save = (double *)malloc(sizeof(double) * 6 * (size_t)n);
  memcpy(save, coords.fxl, sizeof(double) * n);
  memcpy(save + n, coords.fyl, sizeof(double) * n);
  memcpy(save + 2 * n, coords.fzl, sizeof(double) * n);
  memcpy(save + 3 * n, coords.fxs, sizeof(double) * n);
  memcpy(save + 4 * n, coords.fys, sizeof(double) * n);
  memcpy(save + 5 * n, coords.fzs, sizeof(double) * n);
  {
    double vh, v, w, wt[9];
    /* LJ, long level: force_ter(...,1) md_finter.c:110 */
    zero3(coords.fxl, coords.fyl, coords.fzl, n);
    zero3(coords.fxs, coords.fys, coords.fzs, n);
    force_ter(&simparms, &coords, &inter, &ngbr, 1);
    rec_force("f_lj_l", n, coords.fxl, coords.fyl, coords.fzl, coords.amass, 0);
    rec_force("f_lj_s", n, coords.fxs, coords.fys, coords.fzs, coords.amass, 0);
    vh = v = w = 0; for (i = 0; i < 9; i++) wt[i] = 0;
    getsvirter(&vh, &v, &w, wt);
    rec1d("lj_vhinter", vh); rec1d("lj_vinter", v); rec1d("lj_winter", w);
    recd("lj_wtensor", 9, wt);
    /* real-space Ewald, long level: force_ter_e(...,1) md_finter_e.c:78 */
    zero3(coords.fxl, coords.fyl, coords.fzl, n);
    zero3(coords.fxs, coords.fys, coords.fzs, n);
    force_ter_e(&simparms, &coords, &inter, &ngbr, 1);
    rec_force("f_el_l", n, coords.fxl, coords.fyl, coords.fzl, coords.amass, 0);
    rec_force("f_el_s", n, coords.fxs, coords.fys, coords.fzs, coords.amass, 0);
    v = w = 0; for (i = 0; i < 9; i++) wt[i] = 0;
    getsvirter_e(&v, &w, wt);
    rec1d("el_velec", v); rec1d("el_welec", w); recd("el_wtensor", 9, wt);
    if (simparms.iperd == 3 && coords.coul.ncharge > 0) {
      /* reciprocal space: fk_ewald md_ewald.c:185 */
      zero3(coords.fxl, coords.fyl, coords.fzl, n);
      fk_ewald(&simparms, &coords);
      rec_force("f_k", n, coords.fxl, coords.fyl, coords.fzl, coords.amass, 0);
      rec1d("k_vk_ewald", coords.coul.vk_ewald);
      rec1d("k_vp_ewald", coords.coul.vp_ewald);
      recd("k_vp_tensor", 9, coords.coul.vp_ewald_tensor);
      /* excluded-pair correction: ecorr md_ewald.c:385 */
      zero3(coords.fxl, coords.fyl, coords.fzl, n);
      ecorr(&simparms, &coords);
      rec_force("f_ecorr", n, coords.fxl, coords.fyl, coords.fzl, coords.amass, 0);
      rec1d("c_pot_ecorr", coords.coul.pot_ecorr);
      rec1d("c_prs_ecorr", coords.coul.prs_ecorr);
      recd("c_prs_tensor", 9, coords.coul.prs_ecorr_tensor);
    }
    /* short level (RESPA inner nonbonded): force_ter(...,0), force_ter_e(...,0) */
    zero3(coords.fxs, coords.fys, coords.fzs, n);
    force_ter(&simparms, &coords, &inter, &ngbr, 0);
    rec_force("f_lj_short", n, coords.fxs, coords.fys, coords.fzs, coords.amass, 0);
    zero3(coords.fxs, coords.fys, coords.fzs, n);
    force_ter_e(&simparms, &coords, &inter, &ngbr, 0);
    rec_force("f_el_short", n, coords.fxs, coords.fys, coords.fzs, coords.amass, 0);
    /* bonded (inner level): fbond md_fbond.c:76, fbend md_fbend.c:126 */
    zero3(coords.fxa, coords.fya, coords.fza, n);
    fbond(&simparms, &coords);
    rec_force("f_bond", n, coords.fxa, coords.fya, coords.fza, coords.amass, 0);
    zero3(coords.fxa, coords.fya, coords.fza, n);
    fbend(&simparms, &coords);
    rec_force("f_bend", n, coords.fxa, coords.fya, coords.fza, coords.amass, 0);
    /* cross bonds (inner level) and the torsion level: fbondx md_fbocross.c:40,
       ftors md_ftors.c:117, fonfo md_fonefour.c:70 */
    if (coords.bondxs.nbondxs > 0) {
      zero3(coords.fxa, coords.fya, coords.fza, n);
      fbondx(&simparms, &coords);
      rec_force("f_bondx", n, coords.fxa, coords.fya, coords.fza, coords.amass, 0);
    }
    if (coords.tors.ntorss > 0) {
      zero3(coords.fxr, coords.fyr, coords.fzr, n);
      ftors(&simparms, &coords);
      rec_force("f_tors", n, coords.fxr, coords.fyr, coords.fzr, coords.amass, 0);
    }
    if (coords.onfo.n14s > 0) {
      zero3(coords.fxr, coords.fyr, coords.fzr, n);
      fonfo(&simparms, &coords);
      rec_force("f_onfo", n, coords.fxr, coords.fyr, coords.fzr, coords.amass, 0);
    }
  }
  /* restore the state step_init left behind (forces are re-made by step()) */
  force(&simparms, &coords, &inter, &ngbr, 2);
  force(&simparms, &coords, &inter, &ngbr, 3);
  memcpy(coords.fxl, save, sizeof(double) * n);
  memcpy(coords.fyl, save + n, sizeof(double) * n);
  memcpy(coords.fzl, save + 2 * n, sizeof(double) * n);
  memcpy(coords.fxs, save + 3 * n, sizeof(double) * n);
  memcpy(coords.fys, save + 4 * n, sizeof(double) * n);
  memcpy(coords.fzs, save + 5 * n, sizeof(double) * n);
  free(save);

  /* ---- a short trajectory through CM3D's own step() (md_step.c:62) ---- */
  rec1i("nsteps", nsteps);
  if (nsteps > 0) {
    double *eng = (double *)malloc(sizeof(double) * 8 * (size_t)nsteps);
    int s;
    simparms.istep = simparms.istep > 0 ? simparms.istep : 1;
    for (s = 0; s < nsteps; s++, simparms.istep++) {
      step(&simparms, &coords, &energies, &inter, &ngbr);
      geteng(&simparms, &coords, &energies);
      gettngbr(&ngbr);
      eng[8 * s + 0] = energies.poter;
      eng[8 * s + 1] = energies.potra;
      eng[8 * s + 2] = energies.zke;
      eng[8 * s + 3] = energies.vinter;
      eng[8 * s + 4] = energies.velec;
      eng[8 * s + 5] = energies.vewald;
      eng[8 * s + 6] = energies.prsi;
      eng[8 * s + 7] = (double)ngbr.update;
    }
    recd("traj_eng", 8LL * nsteps, eng);
    free(eng);
    recd("final_px", n, coords.px); recd("final_py", n, coords.py);
    recd("final_pz", n, coords.pz);
    recd("final_vx", n, coords.vx); recd("final_vy", n, coords.vy);
    recd("final_vz", n, coords.vz);
    rec_force("final_acc_l", n, coords.fxl, coords.fyl, coords.fzl, coords.amass, 0);
    if (simparms.ntherm > 0) {
      int t;
      double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)simparms.ntherm * simparms.nchain);
      for (t = 0; t < simparms.ntherm; t++) {
        memcpy(buf + (size_t)t * simparms.nchain, coords.eta[t], sizeof(double) * simparms.nchain);
        memcpy(buf + (size_t)(simparms.ntherm + t) * simparms.nchain, coords.veta[t], sizeof(double) * simparms.nchain);
      }
      recd("final_nhc_eta", (long long)simparms.ntherm * simparms.nchain, buf);
      recd("final_nhc_veta", (long long)simparms.ntherm * simparms.nchain, buf + (size_t)simparms.ntherm * simparms.nchain);
      free(buf);
    }
    dump_energies("ef_", &energies);
  }
  fwrite("ENDDUMP!", 1, 8, g_out);
  fclose(g_out);
  return 0;
}
