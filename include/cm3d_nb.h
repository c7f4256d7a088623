/*
 * cm3d_nb.h -- C ABI of the B200 nonbonded force engine for CM3D.
 *
 * The engine replaces CM3D's nonbonded force path: the Verlet/link-cell
 * neighbour lists with minimum image, the tabulated Lennard-Jones and
 * real-space Ewald pair kernels, the reciprocal-space structure-factor sums
 * with the excluded-pair correction, and (so the whole RESPA step can stay on
 * the GPU) the harmonic bond/bend inner level and the velocity/position
 * updates.  Every entry point below names the CM3D routine it replaces
 * (file:line within the CM3D source tree).
 *
 * Conventions
 *   - Only plain C types cross this boundary: pointers, sizes, doubles.
 *   - Arrays follow CM3D's layout: per-atom SoA blocks (px, py, pz ...),
 *     the cell matrix hmat[9] row-major as COORDS.hmat, per-interaction
 *     tables of length ntable stored back to back as INTER.vtab[0].
 *   - Units are CM3D's (K, Angstrom, ps, amu*MCONV, e*sqrt(CCONV)).
 *   - The stored forces are accelerations, as in CM3D after rmass()
 *     (energy/control/md_fcntr.c:74-75).
 *   - Every function returns CM3D_NB_OK (0) or a negative error code; the
 *     message of the last error on the calling thread is available from
 *     cm3d_nb_last_error().  Nothing here exits the process: the CM3D-side
 *     shim turns errors into md_error()/md_warning() as CM3D would.
 *   - A context is single-threaded, like CM3D's own state (module statics
 *     in md_fnopol.c:33, finter_e.c:31, md_finter.c:48); separate contexts
 *     may be driven from separate threads.
 */
#ifndef CM3D_NB_H
#define CM3D_NB_H

#ifdef __cplusplus
extern "C" {
#endif

#define CM3D_NB_OK 0
#define CM3D_NB_ERR_ARG -1        /* invalid argument / unsupported input */
#define CM3D_NB_ERR_CUDA -2       /* CUDA runtime failure */
#define CM3D_NB_ERR_NOMEM -3      /* device allocation failed */
#define CM3D_NB_ERR_STATE -4      /* call out of order (e.g. force before get_ngbr) */
#define CM3D_NB_ERR_OVERFLOW -5   /* a device list outgrew its capacity (engine retries) */
#define CM3D_NB_ERR_NODEV -6      /* no CUDA device */

/* precision modes */
#define CM3D_NB_PLAIN_FP64 0      /* FP64 throughout, pair-per-thread over CM3D's
                                     half lists, atomic force scatter: the plain
                                     one-system-per-launch comparator */
#define CM3D_NB_MIXED 1           /* FP32 distances/tables/phases on
                                     cell-relative coordinates, FP64
                                     accumulation, full lists, no atomics */

/* which force block (COORDS fields) */
#define CM3D_NB_FXL 0             /* fxl,fyl,fzl: long-range nonbonded */
#define CM3D_NB_FXS 1             /* fxs,fys,fzs: short (switched) nonbonded */
#define CM3D_NB_FXA 2             /* fxa,fya,fza: bonds + bends + cross bonds */
#define CM3D_NB_FXR 3             /* fxr,fyr,fzr: torsions + 1-4 pairs */

#define CM3D_NB_MAXPOWER_TORS 7   /* MAXPOWER_TORS (include/md_defines.h:43) */

/* which pair list (NGBR fields) */
#define CM3D_NB_LIST_T 0          /* inpt/jnpt:   LJ, r^2 < rmaxl_skin2[intr] */
#define CM3D_NB_LIST_S 1          /* inps/jnps:   LJ, r^2 < rmaxs_skin2[intr] */
#define CM3D_NB_LIST_TE 2         /* inpte/jnpte: charged, r^2 < rmaxl_skin2_e */
#define CM3D_NB_LIST_SE 3         /* inpse/jnpse: charged, r^2 < rmaxs_skin2_e */

/*
 * System description.  Field names follow CM3D's structs so the shim can fill
 * it straight from SIMPARMS / COORDS / INTER / COUL / BONDS / BENDS
 * (include/md_typedef.h:59-268).  All pointers are host memory and are only
 * read during cm3d_nb_create(); the engine keeps device copies.
 */
typedef struct cm3d_nb_system {
  /* SIMPARMS (md_typedef.h:120) */
  int natoms;
  int iperd;                 /* periodicity; the engine requires 3 */
  int nres_lrf;              /* SIMPARMS.ninter */
  int nres_intra;            /* SIMPARMS.ninnra */
  int nres_tors;             /* SIMPARMS.ninrra */
  int ndof;
  double dt;                 /* ps (after TCONV) */
  double vlrc, wlrc;         /* long-range corrections (md_searchbase.c:212-235) */
  /* COORDS (md_typedef.h:201) */
  double hmat[9];
  const double *px, *py, *pz;
  const double *vx, *vy, *vz;
  const double *amass;
  const double *qch;
  /* INTER (md_typedef.h:255) */
  int ntypes;                /* atom types */
  const int *itype;          /* [natoms] */
  const int *map;            /* [ntypes*ntypes], interaction index or -1 (null) */
  int ninter;                /* INTER.ntype: non-null interactions */
  int ntable;
  const double *vtab;        /* [ninter*ntable] V */
  const double *dvtab;       /* [ninter*ntable] (dV/dr)/r */
  const double *switchs;     /* [ninter*ntable] RESPA switch */
  const double *rmaxs_cut2, *rmins_cut2, *rmaxl_cut2, *rminl_cut2;
  const double *rmaxs_skin2, *rmaxl_skin2, *dx2tab;     /* [ninter] */
  double skin_ter, rheal;
  const double *coultab, *dcoultab, *switchse;          /* [ntable]; NULL if no charges */
  double dx2coul, rmins_coul2, rmaxs_coul2, rminl_coul2, rmaxl_coul2;
  double rmaxs_skin2_e, rmaxl_skin2_e;
  const int *excl_off, *excl_idx;   /* INTER.nexclude/exclude as CSR: atom i's
                                       sorted list is excl_idx[excl_off[i]..excl_off[i+1]) */
  /* COUL (md_typedef.h:59) */
  const int *cexcl_off, *cexcl_idx; /* COUL.nexclude/exclude as CSR */
  int ktot;
  const int *ka, *kb, *kc;          /* k-vectors in CM3D's order (md_ewald.c:93-114) */
  double kappa, falp2, ewald_self, ewald_bkg;
  int necorr;
  const int *iecorr, *jecorr;
  /* BONDS / BENDS (md_typedef.h:71-79); harmonic forms only */
  int nbonds, nbond_types;
  const int *ibond, *jbond, *idxbond, *itypbond;
  const double *eqbond, *fkbond;
  int nbends, nbend_types;
  const int *ibend, *jbend, *kbend, *idxbend, *itypbend;
  const double *eqbend, *fkbend;
  /* TORS / ONFO / BONDXS (md_typedef.h:81-100).  Torsions and 1-4 pairs
     make the torsion RESPA level (force level 3 into fxr: ftors
     md_ftors.c:117, fonfo md_fonefour.c:70); cross bonds join the bonds and
     bends of level 2 (fbondx md_fbocross.c:40). */
  int ntors, n14, nbondx;
  int ntors_types;                            /* TORS.itypes */
  const int *itors, *jtors, *ktors, *ltors;   /* [ntors] */
  const int *idxtors;                         /* [ntors] torsion type */
  const int *tors_ind_pot;                    /* [ntors_types] form: 0 harmonic in phi,
                                                 1 cosine power series (2, cosine
                                                 with phases, is refused) */
  const int *tors_ind_pot_num;                /* [ntors_types] row of eqtors/fktors (form 0)
                                                 or of vphi (form 1) */
  int ntors_harm;                             /* rows of eqtors / fktors */
  const double *eqtors, *fktors;
  int ntors_series;                           /* rows of vphi */
  const double *vphi;                         /* [ntors_series * CM3D_NB_MAXPOWER_TORS] */
  int n14_types, n14table;
  const int *i14, *j14, *i14dx;               /* [n14] atoms and 1-4 type */
  const double *r14min2, *r14max2, *dx214tab; /* [n14_types] table ranges (squared) */
  const double *v14tab, *dv14tab;             /* [n14_types * n14table] V and (dV/dr)/r */
  double scale_onefour, scale_onefour_e;
  int nbondx_types;
  const int *ibondx, *jbondx, *kbondx, *idxbondx;   /* [nbondx] */
  const double *eq1bondx, *eq2bondx, *fkbondx;      /* [nbondx_types] */
  /* frozen atoms (SIMPARMS.nfreeze, COORDS.ifreeze): every force level ends
     with their velocities and forces set to zero (freeze_atom
     md_fcntr.c:311-329) */
  int nfreeze;
  const int *ifreeze;
  /* SIMPARMS.iensemble / ntherm / nchain and COORDS' Nose-Hoover chain state
     (md_typedef.h:122-125, 203-224; set_therm_new md_therm.new.c:32), as
     samveta leaves it.  iensemble 0 (NVE, no thermostats) or 1 (NVT: the
     chains integrated by intnhc_new, md_therm.new.c:278, inside the inner
     level of step()); cm3d_nb_create refuses anything else (barostats).
     Every system of a batch has the same ensemble and chain length. */
  int iensemble, ntherm, nchain;
  const int *ithm;                            /* [natoms] thermostat of each atom (-1: none) */
  const double *mnh, *gkt, *nhc_eta, *nhc_veta;   /* [ntherm * nchain] */
} cm3d_nb_system;

typedef struct cm3d_nb_options {
  int device;                /* CUDA device ordinal */
  int mode;                  /* CM3D_NB_PLAIN_FP64 or CM3D_NB_MIXED */
  int need_short;            /* 1: always produce fxs at level 1 (CM3D does);
                                0: only when nres_lrf > 1 (fxs is multiplied by
                                dter1 = 0 otherwise, md_step.c:78,99) */
  int tpa;                   /* mixed pair kernel: lanes per atom (0 = auto) */
  int use_graph;             /* capture cm3d_nb_step() in a CUDA graph */
  double cell_scale;         /* list-build cells at least cell_scale list radii
                                wide (>= 1; 0 or below 1 means 1): fewer, larger
                                cells -- larger windows per pair-kernel block,
                                more candidates per atom in the list build */
} cm3d_nb_options;

/* energies/virials collected as getvireal()+geteng() do (md_fcntr.c:136-308) */
typedef struct cm3d_nb_energies {
  double vinter, vhinter, winter, wintertensor[9];   /* getsvirter  md_fnopol.c:386 */
  double velec, welec, welectensor[9];               /* getsvirter_e finter_e.c:410 */
  double vewald, wewald, wewaldtensor[9];            /* getvewald   md_ewald.c:364 */
  double vbond, vbend, wbond, wbend;
  double US, U, W, Wtensor[9];
  double zke, p2m_tensor[9];                         /* get_p2mt md_fcntr.c:332 */
  double prsi, prs_tensor[9], tiout, poter, poth, potra;
  /* torsion level and cross bonds: getvtors md_ftors.c:296, getvonfo
     md_fonefour.c:160, getvbondx md_fbocross.c:100 (which adds the cross
     bonds' energy and virial to vbond / wbond); UI, WI and WItensor sum the
     intramolecular terms as getvireal does (md_fcntr.c:206-215) */
  double vtors, wtors, vonfo, vonfo_e, wonfo, wonfo_e;
  double UI, WI, WItensor[9];
} cm3d_nb_energies;

typedef struct cm3d_nb_status_t {
  long long table_underflow;  /* pairs below the table start (md_fnopol.c:133-140) */
  long long rebuilds;         /* neighbour-list rebuilds so far */
  long long resets;           /* RESETPOS events (md_finter.c:79-95) */
  long long overflows;        /* list-capacity overflows handled by regrowth */
  int nonfinite;              /* a NaN/Inf reached the forces or energies */
  int last_istep;
  int stage_timeouts;         /* pair-kernel blocks whose window copies did not
                                 complete within the wait limit (their work was
                                 not done: the step's results are invalid);
                                 0 in every run so far */
} cm3d_nb_status_t;

typedef struct cm3d_nb_ctx cm3d_nb_ctx;

/* ------------------------------------------------------------ library */
int cm3d_nb_version(void);
const char *cm3d_nb_last_error(void);
int cm3d_nb_device_count(int *count);
void cm3d_nb_default_options(cm3d_nb_options *opt);

/* ------------------------------------------------------------ context */
/* Upload a system; replaces the allocations CM3D makes in read_parmfile /
   allocate_lists / set_charges (md_readparm.c:35, ngbr_list.c:584,
   elec_ngbr.c:36).  Lists are not built until cm3d_nb_get_ngbr(). */
int cm3d_nb_create(const cm3d_nb_system *sys, const cm3d_nb_options *opt,
                   cm3d_nb_ctx **out);
void cm3d_nb_destroy(cm3d_nb_ctx *ctx);

/* ------------------------------------------------------------ batches */
/* Many independent systems in one context (no CM3D counterpart: CM3D runs one
   system per process).  Each system keeps its own box, cell grid, tables,
   k-vectors, neighbour lists, rebuild decisions (nrefsh with RESETPOS) and
   energies, exactly as it would alone; every kernel of a step covers all
   systems at once.  The systems' atoms are concatenated in array order, so
   the per-atom calls below (positions, velocities, forces) see
   sum(natoms) atoms and system s owns [first, first + natoms) of them.
   Requirements: the mixed engine, and the same ntable, dt and RESPA levels
   (nres_lrf / nres_tors / nres_intra) in every system.  cm3d_nb_create is
   cm3d_nb_create_batch with nsys = 1; the single-system routines below
   report system 0. */
int cm3d_nb_create_batch(const cm3d_nb_system *systems, int nsys,
                         const cm3d_nb_options *opt, cm3d_nb_ctx **out);
int cm3d_nb_num_systems(cm3d_nb_ctx *ctx, int *nsys);
int cm3d_nb_system_atoms(cm3d_nb_ctx *ctx, int sys, int *first, int *natoms);
/* getvireal()+geteng() of one system / of every system (e[nsys]) */
int cm3d_nb_get_system_energies(cm3d_nb_ctx *ctx, int sys, cm3d_nb_energies *e);
int cm3d_nb_get_all_energies(cm3d_nb_ctx *ctx, cm3d_nb_energies *e);
/* per-system list rebuilds and RESETPOS events since creation (arrays of nsys) */
int cm3d_nb_system_counts(cm3d_nb_ctx *ctx, long long *rebuilds, long long *resets);
/* NVT: system sys's Nose-Hoover chain positions and velocities (COORDS.eta,
   veta, md_typedef.h:224), ntherm x nchain each, as the steps left them;
   *ntherm and *nchain receive the sizes (0 for an NVE context) */
int cm3d_nb_get_nhc(cm3d_nb_ctx *ctx, int sys, double *eta, double *veta, int *ntherm, int *nchain);

/* host <-> device state (COORDS.px..pz, vx..vz, hmat) */
int cm3d_nb_set_positions(cm3d_nb_ctx *ctx, const double *px, const double *py,
                          const double *pz);
int cm3d_nb_get_positions(cm3d_nb_ctx *ctx, double *px, double *py, double *pz);
/* a new box matrix (COORDS.hmat, row-major) for a one-system context, as
   CM3D's barostats (intbar, integrate/md_baro.c:72) change it between force
   calls: H^-1, the volume and every box-derived parameter follow.  The cell
   grid keeps its counts: a box that shrinks below it (a cell narrower than
   the list radius) returns CM3D_NB_ERR_STATE, and a new context is needed. */
int cm3d_nb_set_box(cm3d_nb_ctx *ctx, const double hmat[9]);
int cm3d_nb_set_velocities(cm3d_nb_ctx *ctx, const double *vx, const double *vy,
                           const double *vz);
int cm3d_nb_get_velocities(cm3d_nb_ctx *ctx, double *vx, double *vy, double *vz);
int cm3d_nb_get_forces(cm3d_nb_ctx *ctx, int which, double *fx, double *fy,
                       double *fz);
int cm3d_nb_set_forces(cm3d_nb_ctx *ctx, int which, const double *fx,
                       const double *fy, const double *fz);

/* ------------------------------------------------- CM3D entry points */
/* get_ngbr()        energy/control/ngbr_list.c:297 (with get_ngbr_e,
                     elec_ngbr.c:220): rebuild all four lists from the
                     current positions and snapshot them into dxn. */
int cm3d_nb_get_ngbr(cm3d_nb_ctx *ctx);
/* nrefsh()          energy/control/md_finter.c:43: rebuild when any atom
                     moved more than skin/2, with the RESETPOS pull-back
                     when the previous rebuild is fewer than 3 steps old. */
int cm3d_nb_nrefsh(cm3d_nb_ctx *ctx, int istep, int *rebuilt);
/* force()           energy/control/md_fcntr.c:44 for iflg 0 (short
                     nonbonded), 1 (full nonbonded + Ewald), 2 (bonds, bends
                     and cross bonds) and 3 (torsions and 1-4 pairs); results
                     stored as accelerations. */
int cm3d_nb_force(cm3d_nb_ctx *ctx, int iflg);
/* force_ter()       energy/control/md_finter.c:110 -> force_npol()
                     energy/inter/md_fnopol.c:46: LJ over the t (iflg 1) or
                     s (iflg 0) list; adds raw forces to fxl/fxs (iflg 1) or
                     fxs (iflg 0) and resets the LJ accumulators (zero_potl). */
int cm3d_nb_force_ter(cm3d_nb_ctx *ctx, int iflg);
/* force_ter_e()     energy/control/md_finter_e.c:78 -> force_e()
                     energy/inter/finter_e.c:42: real-space Ewald over the te
                     (iflg 1) or se (iflg 0) list. */
int cm3d_nb_force_ter_e(cm3d_nb_ctx *ctx, int iflg);
/* fk_ewald()        energy/inter/md_ewald.c:185: structure factors,
                     reciprocal energy/virial, adds forces to fxl. */
int cm3d_nb_fk_ewald(cm3d_nb_ctx *ctx);
/* ecorr()           energy/inter/md_ewald.c:385: excluded-pair correction,
                     adds forces to fxl. */
int cm3d_nb_ecorr(cm3d_nb_ctx *ctx);
/* zero a force block / rmass() utils/md_util.new.c:219 on it */
int cm3d_nb_zero_forces(cm3d_nb_ctx *ctx, int which);
int cm3d_nb_rmass(cm3d_nb_ctx *ctx, int which);
/* getsvirter()      energy/inter/md_fnopol.c:386 (adds, as CM3D does) */
int cm3d_nb_getsvirter(cm3d_nb_ctx *ctx, double *vhinter, double *vinter,
                       double *winter, double wintert[9]);
/* getsvirter_e()    energy/inter/finter_e.c:410 */
int cm3d_nb_getsvirter_e(cm3d_nb_ctx *ctx, double *velec, double *welec,
                         double welectensor[9]);
/* getvewald()       energy/inter/md_ewald.c:364 */
int cm3d_nb_getvewald(cm3d_nb_ctx *ctx, double *pot_ewald, double *prs_ewald,
                      double prs_ewald_tensor[9]);
/* step_init()       integrate/md_step.c:32: lists, forces at levels 1 and 2,
                     energies. */
int cm3d_nb_step_init(cm3d_nb_ctx *ctx);
/* step()            integrate/md_step.c:62, nsteps times starting at
                     SIMPARMS.istep = istep0 (NVE, or NVT with the Nose-Hoover
                     chains of cm3d_nb_system; a barostat stays with CM3D's
                     host integrator, the engine following its box through
                     cm3d_nb_set_box). */
int cm3d_nb_step(cm3d_nb_ctx *ctx, int istep0, int nsteps);
/* The same steps without waiting (no CM3D counterpart): cm3d_nb_step_async
   launches them on the context's stream and returns, so that several
   contexts' steps overlap on the device; cm3d_nb_step_query reports (*done)
   whether they have completed, without blocking; cm3d_nb_step_wait blocks
   until they have.  Every other call on the context first waits for them.
   (Graph mode; with use_graph = 0 the steps run to completion at once.) */
int cm3d_nb_step_async(cm3d_nb_ctx *ctx, int istep0, int nsteps);
int cm3d_nb_step_query(cm3d_nb_ctx *ctx, int *done);
int cm3d_nb_step_wait(cm3d_nb_ctx *ctx);
/* A host loop that owns the positions and velocities (CM3D's, which reads
   them after every step) without a round trip per array (no CM3D
   counterpart).  cm3d_nb_set_host_outputs registers page-locked host
   buffers (cudaMallocHost / cudaHostRegister; 3 natoms doubles each, x | y |
   z blocks, either may be NULL; NULL for both stops it): every later step
   copies its final positions there as soon as they are final -- on a
   separate stream, beside the step's list build and forces -- and its
   velocities at its end, complete when the step call returns.
   cm3d_nb_step_host copies pos_in and vel_in (x | y | z blocks, page-locked
   for an asynchronous copy; either may be NULL to keep the device's) to the
   device and runs one step (SIMPARMS.istep = istep0).  The input and output
   buffers may be the same. */
int cm3d_nb_set_host_outputs(cm3d_nb_ctx *ctx, double *pos_out, double *vel_out);
int cm3d_nb_step_host(cm3d_nb_ctx *ctx, int istep0, const double *pos_in, const double *vel_in);
/* getvireal(...,1)+geteng() md_fcntr.c:136,259 from the device accumulators */
int cm3d_nb_get_energies(cm3d_nb_ctx *ctx, cm3d_nb_energies *e);

/* pair lists in CM3D's NGBR form: pairs (i, j) of atom indices */
int cm3d_nb_list_count(cm3d_nb_ctx *ctx, int which, long long *npairs);
int cm3d_nb_get_list(cm3d_nb_ctx *ctx, int which, int *ip, int *jp,
                     long long capacity, long long *npairs);

int cm3d_nb_get_status(cm3d_nb_ctx *ctx, cm3d_nb_status_t *st);
int cm3d_nb_synchronize(cm3d_nb_ctx *ctx);
/* the CUDA stream every kernel of this context runs on (cudaStream_t) */
void *cm3d_nb_stream(cm3d_nb_ctx *ctx);

/* --------------------------------------------------------- timing */
/* Bracket every launch of kernel class `cls` with CUDA events on the
   context's stream; cm3d_nb_kernel_time returns the summed device time in
   ms and the number of launches since timing was enabled.
   cls: 0 = pair kernel(s), 1 = k-space, 2 = list build, 3 = integrate
   (enable bit 0; these launches then run eagerly, outside CUDA graphs),
   4 = whole steps of cm3d_nb_step (enable bit 1; graph replays included). */
int cm3d_nb_enable_timing(cm3d_nb_ctx *ctx, int enable);
int cm3d_nb_kernel_time(cm3d_nb_ctx *ctx, int cls, double *ms, long long *launches);
/* number of kernel launches this context issued so far */
long long cm3d_nb_launch_count(cm3d_nb_ctx *ctx);
/* FMA throughput of `device` measured with a dependency-chain probe
   (TFLOP/s, an FMA counted as 2 flops): the roofline denominators of the
   CUDA-core pair and k-space kernels.  No CM3D counterpart. */
int cm3d_nb_measure_peaks(int device, double *fp32_tflops, double *fp64_tflops);
/* Autotuner of the mixed pair kernel (no CM3D counterpart): times the fused
   LJ + real-space Ewald kernels (below) with 4, 8, 16 and 32 lanes per atom
   on the context's current lists (reps launches each, CUDA events), keeps
   the fastest, and recomputes force(1) so the state is as before.  Call
   after cm3d_nb_get_ngbr or cm3d_nb_step_init.  ms_per_launch[4] (may be
   NULL) receives, per lanes-per-atom choice, the time of the faster kernel. */
int cm3d_nb_autotune(cm3d_nb_ctx *ctx, int reps, int *tpa_chosen, double ms_per_launch[4]);
/* The mixed pair kernels (no CM3D counterpart).  GATHER: lane groups read
   j-atoms from global memory; any context can run it.  WINDOW: one system
   with >= 3 cells per axis; a block stages the 27 cells around an i-cell in
   shared memory.  SYSTEM: a batch whose largest system fits in shared memory;
   a block stages the whole system it works on.  COMPACT: one system with >= 3
   cells per axis at the full force level (no RESPA switch copy); its list is
   rewritten after each rebuild as 16-bit indices into the i-cell's staged
   27-cell window, and its tables are replicated across the shared-memory
   banks.  In a batch the compact path covers the systems with >= 3 cells
   per axis, 32 lanes per atom (COMPACT) or, where cells hold a few tens of
   atoms, 8 lanes per atom with several cells in flight per block
   (COMPACT8, when the autotuner finds it faster; CM3D_NB_CW_ROW=8 in the
   environment at create starts there).
   CM3D_NB_PAIR_KERNEL=window keeps a context off the compact kernel.
   cm3d_nb_autotune times the gather kernel and the staged and compact ones
   that apply at every lanes-per-atom choice, keeps the fastest, and
   ms_per_launch[k] is the faster at that choice.  CM3D_NB_PAIR_KERNEL=list in the environment at cm3d_nb_create
   keeps a context on the gather kernel.  cm3d_nb_pair_kernel reports the
   kernel of the last pair launch and the lanes per atom. */
#define CM3D_NB_PAIR_GATHER 0
#define CM3D_NB_PAIR_WINDOW 1
#define CM3D_NB_PAIR_SYSTEM 2
#define CM3D_NB_PAIR_COMPACT 3
#define CM3D_NB_PAIR_COMPACT8 4   /* a batch's compact lists with 8 lanes per atom (small cells) */
int cm3d_nb_pair_kernel(cm3d_nb_ctx *ctx, int *kernel, int *tpa);
/* the cell grid of system `sys` (cells per box direction) and, for the
   compact path, the parts each cell's atoms are split into (work items per
   cell; 1 elsewhere) and the threads of its blocks (0 without it) */
int cm3d_nb_grid(cm3d_nb_ctx *ctx, int sys, int nc[3], int *nsplit, int *block_threads);

/* ------------------------------------------- no-allocation variant */
#define CM3D_NB_NOALLOC_MAX_CHARGES 32768   /* charged atoms per call */
#define CM3D_NB_NOALLOC_MAX_KMAX 15         /* kmax per call (7073 k-vectors) */
/* fk_ewald() (energy/inter/md_ewald.c:185-348) in one call that allocates no
   device memory.  It has no counterpart in the reference, whose fk_ewald
   works on the COORDS arrays that CM3D's set-up allocated; it is for callers
   that cannot allocate device memory at the point where they need the
   reciprocal-space forces: a host program whose own memory pool has already
   reserved the device (several systems packed on one GPU, each in its own
   slice), or one that must not let an allocation stall the device in the
   middle of a time step.  Such a caller owns every input and output buffer;
   no engine context (cm3d_nb_create, which allocates) is involved.

   The call runs the mixed-precision k-space kernels of cm3d_nb_fk_ewald (FP32
   phases from fixed-point fractional coordinates, FP64 sums) on a scratch
   area of about 2.9 MiB that is part of the library's static device memory,
   one per device.  Limits: ncharge <= CM3D_NB_NOALLOC_MAX_CHARGES and
   kmax <= CM3D_NB_NOALLOC_MAX_KMAX; larger inputs return CM3D_NB_ERR_ARG
   (cm3d_nb_fk_ewald has no such limit).

   The first call on a device does a one-time set-up: it looks the scratch
   area up (the CUDA runtime may load the library's device code at that
   moment, which is when the static area itself is reserved) and raises the
   force kernel's shared-memory limit.  Make that first call before any stream
   capture and where a one-time cost is acceptable.  A set-up that fails is
   not remembered: the next call on that device tries it again.  Every call
   launches six kernels on `stream` and returns without waiting for them.

   Where the k-vectors are split over several blocks per atom, the forces
   are summed with FP64 atomic adds whose order varies: two calls on the
   same inputs agree to summation-order rounding (far inside the mixed
   engine's 1e-5 relative bound, as tests/test_zz_no_alloc.py checks), not
   bit for bit.  The energies and virials are summed in a fixed order.

   The call clears the scratch accumulators itself; nothing has to start at
   zero except what the caller wants in fxl, to which the forces are added.
   Two calls on one device whose work overlaps in time (different streams,
   or different host threads) share the scratch area and race: serialise
   them, e.g. on one stream.

   device         CUDA ordinal; made current for the call, the caller's
                  current device is restored before returning
   stream         cudaStream_t to launch on (NULL: the default stream)
   natoms, pos    device, 3*natoms doubles: px | py | pz (COORDS.px ...)
   q              device, natoms charges (COORDS.qch)
   ncharge, icharge  device, the charged atoms' indices (COUL.icharge)
   hmat           host, the cell matrix (COORDS.hmat)
   kmax           ewald_setup's k-vector set (md_ewald.c:93-114)
   falp2, ewald_self, ewald_bkg   COUL.falp2 / ewald_self / ewald_bkg
                  (md_ewald.c:59-76)
   fxl            device, 3*natoms doubles: the forces are ADDED, as fk_ewald
                  adds them to COORDS.fxl
   out            device, 11 doubles, overwritten: vk_ewald, vp_ewald,
                  vp_ewald_tensor[9] (md_ewald.c:336-348) */
int cm3d_nb_fk_ewald_noalloc(int device, void *stream, int natoms,
                             const double *pos, const double *q, int ncharge,
                             const int *icharge, const double hmat[9],
                             int kmax, double falp2, double ewald_self,
                             double ewald_bkg, double *fxl, double *out);

/* ------------------------------------------ host set-up restatements */
/* One interaction's LJ table, as get_ter_parm() builds it
   (input/md_getparm.c:236-237, 321-366 with func_lj md_funcvdw.c:40):
   ntable points uniform in r^2 from rmin^2; V, (dV/dr)/r and the cubic
   RESPA switch over [rres-rheal, rres].  `shift` subtracts V[ntable-3]
   (md_searchbase.c:181-188).  Outputs are ntable long; *dx2tab is set. */
int cm3d_nb_lj_table(double eps, double sig, double rmin, double rmax,
                     double rres, double rheal, double skin, int ntable,
                     int shift, double *vtab, double *dvtab, double *switchs,
                     double *dx2tab);
/* The real-space Ewald table of set_charges() (elec_ngbr.c:51-103 with
   func_kerf md_funcvdw.c:219; func_coul when iperd != 3). */
int cm3d_nb_coul_table(double alpha, double rcute_min, double rcute_resp,
                       double rcute_max, double rheal, double skin, int ntable,
                       int iperd, int shift, double *coultab, double *dcoultab,
                       double *switchse, double *dx2coul);
/* The half-space spherical k-vector set of ewald_setup() (md_ewald.c:93-114);
   with ka == NULL only *ktot is returned. */
int cm3d_nb_ewald_kvectors(int kmax, int *ka, int *kb, int *kc, int *kup,
                           int *ktot);

#ifdef __cplusplus
}
#endif
#endif /* CM3D_NB_H */
