// nb_common.cuh -- engine context and helpers shared by the CUDA sources.
//
// Device layout (one system per context):
//   pos, vel, fxl, fxs, fxa     3N doubles each, x | y | z blocks, original
//                               atom order -- the layout of CM3D's contiguous
//                               COORDS blocks (utils/md_util.new.c:113-141)
//   acc[]                       FP64 energy/virial accumulators (ACC_* below)
//   cell grid + sorted arrays   rebuilt with the lists (nb_list.cu)
//   half lists t/s/te/se        CM3D's NGBR lists as (i, j) pairs
//   full list (mixed mode)      per sorted atom, packed 32-bit entries
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/cm3d_nb.h"

namespace cm3d {

// ------------------------------------------------------------ accumulators
enum {
  ACC_SPOTL = 0,          // sum V_LJ                     (md_fnopol.c spotl)
  ACC_SPOTHL = 1,         // sum V_LJ - V(ntable-4)       (spothl)
  ACC_SPRSL = 2,          // sum -r^2 f                   (sprsl)
  ACC_SPRSLT = 3,         // 9: LJ virial tensor          (sprslt)
  ACC_SPOTE = 12,         // elec energy                  (finter_e.c spote)
  ACC_SPOTHE = 13,        // shifted elec energy          (spothe)
  ACC_SPRSE = 14,         // elec virial                  (sprse)
  ACC_SPRSET = 15,        // 9: elec virial tensor        (sprset)
  ACC_VK = 24,            // sum preg |S|^2               (fk_ewald vk)
  ACC_VP = 25,            // sum prep |S|^2 g2            (vp)
  ACC_VPT = 26,           // 9: reciprocal virial tensor  (vp_tensor)
  ACC_POT_ECORR = 35,     // md_ewald.c ecorr spot
  ACC_PRS_ECORR = 36,     // ecorr sprs
  ACC_PRS_ECORRT = 37,    // 9
  ACC_VBOND = 46,         // getvbond energy
  ACC_WBOND = 47,         // getvbond virial
  ACC_WBONDT = 48,        // 9
  ACC_VBEND = 57,         // getvbend energy
  ACC_P2MT = 58,          // 9: get_p2mt kinetic tensor
  ACC_WBEND = 67,         // getvbend virial (md_fbend.c compiles it with PRESSURE)
  ACC_WBENDT = 68,        // 9
  ACC_VTORS = 77,         // getvtors energy (its virial is the tensor's trace)
  ACC_WTORST = 78,        // 9: torsion virial tensor (md_ftors.c PRESSURE)
  ACC_VONFO = 87,         // getvonfo: tabulated 1-4 energy (unscaled)
  ACC_VONFO_E = 88,       //           1-4 Coulomb energy (unscaled)
  ACC_WONFO = 89,         //           tabulated 1-4 virial (unscaled)
  ACC_WONFOT = 90,        // 9
  ACC_WONFOET = 99,       // 9: 1-4 Coulomb virial tensor (unscaled)
  ACC_WBONDXT = 108,      // 9: getvbondx tensor (its energy and virial go to ACC_VBOND/WBOND)
  ACC_COUNT = 117,
  // each system owns ACC_STRIDE doubles of acc[]: its accumulators, then
  // device copies of its H^-1 (ACC_COUNT..+9) and H (+9..+18)
  ACC_STRIDE = 144
};

// Per-system parameters of a context that holds several independent systems
// (a batch), one entry per system in a device array.  The systems' atoms are
// concatenated: system s owns atoms [a0, a0 + n), in original order and in
// cell-sorted order alike, cells [c0, c0 + ncells), charged atoms
// icharge[q0 .. q0 + nq) and k rows / k-vectors / tiles as below.
struct SysP {
  int a0, n;
  int c0, ncells, nc[3];
  int nsx, nsy, nsz, sx[3], sy[3], sz[3];   // unique stencil offsets per axis
  int ntypes, map0;          // type map at map[map0 ...], ntypes^2 global interaction indices
  int inter0, ninter;        // its interactions: global indices [inter0, inter0 + ninter)
  int coul;                  // Coulomb table index (tables at coul * ntable), -1: no charges
  int smallbox;              // box narrower than two list radii: minimum image per pair
  int excl, cexcl;           // the system has LJ / Coulomb exclusions (0: the list tests skip them)
  int q0, nq;
  int krow0, nrows, kk0, ktot;   // k rows and k-vectors (global indices)
  int ktile0, ktiles;        // structure-factor tiles (global tile ids)
  int ftile0, ftiles;        // reciprocal-force tiles (global tile ids)
  long long spart0;          // first per-tile partial S(k) of the system
  float lim2;                // FP32 list prefilter radius^2 (inf = off)
  float rc2_el, dx2c, offc, tablast_e;
  float hF[9], hiF[9];
  double h[9], hi[9];
  double rmaxl_skin2_e, rmaxs_skin2_e;   // -1 without charges
  double skin2q;             // (skin / 2)^2
  double near_s[3];          // small boxes: |fractional displacement| above which a listed pair
                             // may change its nearest image before the next rebuild
  double falp2, rvol, kappa, kappa2;
  float4 shift[27];          // cell-corner shifts H k / nc, k in {-1, 0, 1}^3 (FP32 hi part)
  float4 shift_lo[27];       // their FP32 residuals (shift + shift_lo = the FP64 shift)
};
// device status words (long long)
enum {
  ST_UNDERFLOW = 0,       // table underflows (k < 1)
  ST_NONFINITE = 1,
  ST_OVERFLOW = 2,        // a list fill ran past its capacity
  ST_RESETS = 3,          // RESETPOS events
  ST_REBUILDS = 4,
  ST_BADSHIFT = 5,        // a pair's cell shift fell outside the 27-entry table
  ST_NEED_STRIDE = 6,     // longest full list that did not fit its slot
  ST_CWIN = 7,            // a cell window too large for the compact list (nb_cwin.cu)
  ST_STAGE_TIMEOUT = 8,   // a window's bulk copies not complete within the wait limit (nb_cwin.cu)
  ST_COUNT = 9
};
// device integer state
enum {
  IS_ISTEP = 0,           // SIMPARMS.istep of the step being taken
  IS_ISTEPLAST = 1,       // md_finter.c:48 static isteplast
  IS_REBUILD = 2,         // rebuild requested by the displacement check
  IS_HALT = 3,            // a device-side rebuild outgrew a list: the rest
                          // of the captured step does nothing, the host
                          // grows the buffers and finishes the step
  IS_INTR = 4,            // RESPA level (intr) the step is in
  IS_COUNT = 8
};

// Gate of kernels that run inside a captured step: with gs == nullptr (host
// driven) never skip; otherwise skip once the step is halted, and list-build
// kernels (need_rebuild) also when no rebuild was requested.
__device__ __forceinline__ bool gated_off(const int *gs, int need_rebuild) {
  return gs && (gs[IS_HALT] != 0 || (need_rebuild && gs[IS_REBUILD] == 0));
}
// per-system counters (sstat[s * SS_COUNT + ...])
enum { SS_REBUILDS = 0, SS_RESETS = 1, SS_COUNT = 2 };

// Sum NV per-thread values into the accumulators of each thread's system
// (acc + sys * ACC_STRIDE + slots[k]).  A warp whose threads all belong to
// one system reduces first and adds once; a mixed warp adds per thread.
// Threads with sys < 0 contribute nothing.  Every thread of the warp calls it.
template <int NV>
__device__ __forceinline__ void sys_acc(double (&v)[NV], int sys, double *acc, const int *slots) {
  const unsigned full = 0xffffffffu;
  const int s0 = __shfl_sync(full, sys, 0);
  if (__all_sync(full, sys == s0 || sys < 0)) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      // a quantity that is zero on every thread (e.g. no bonds in an LJ
      // system) costs one vote, not a reduction
      if (!__any_sync(full, sys >= 0 && v[k] != 0.0)) continue;
      double s = sys < 0 ? 0.0 : v[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(full, s, o);
      if ((threadIdx.x & 31) == 0 && s != 0.0 && s0 >= 0) atomicAdd(acc + (size_t)s0 * ACC_STRIDE + slots[k], s);
    }
  } else if (sys >= 0) {
#pragma unroll
    for (int k = 0; k < NV; k++)
      if (v[k] != 0.0) atomicAdd(acc + (size_t)sys * ACC_STRIDE + slots[k], v[k]);
  }
}

// list totals (long long) written by the list builder
enum { LT_T = 0, LT_S = 1, LT_TE = 2, LT_SE = 3, LT_FULL = 4, LT_COUNT = 5 };

// packed full-list entry (mixed mode): j (sorted index) | shift code | flags
constexpr int ENT_JBITS = 22;
constexpr uint32_t ENT_JMASK = (1u << ENT_JBITS) - 1;
constexpr int ENT_CODE_SHIFT = 22;          // 5 bits: 27 cell-shift codes
constexpr uint32_t ENT_LJ = 1u << 27;       // pair is in CM3D's t list
constexpr uint32_t ENT_EL = 1u << 28;       // pair is in CM3D's te list
constexpr uint32_t ENT_LJS = 1u << 29;      // pair is in CM3D's s list
constexpr uint32_t ENT_ELS = 1u << 30;      // pair is in CM3D's se list
constexpr uint32_t ENT_NEAR = 1u << 31;     // small box: the pair may change image, check it
constexpr int MAX_ATOMS_MIXED = 1 << ENT_JBITS;

// classes 0 pair, 1 k-space, 2 list build, 3 integrate (per kernel, eager
// launches only); 4 whole steps (around graph replays too)
constexpr int NTCLS = 5;
struct Timing {
  bool on = false;          // per-kernel classes 0-3
  bool steps = false;       // class 4
  double ms[NTCLS] = {0, 0, 0, 0, 0};
  long long launches[NTCLS] = {0, 0, 0, 0, 0};
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending[NTCLS];
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
};

// host-side facts of one system of a batch (energies, set-up)
struct SysH {
  int n = 0, ncharge = 0, ndof = 1, ntypes = 0, ninter = 0, ktot = 0, iperd = 3;
  double hmat[9], hmati[9];
  double vlrc = 0, wlrc = 0, ewald_self = 0, ewald_bkg = 0;
  double scale14 = 1, scale14e = 1;   // ONFO.scale_onefour / scale_onefour_e
  double rlist = 0;          // largest list radius (LJ or charges, with skin)
  double skin = 0;           // INTER.skin_ter
  double rmaxl_coul2 = 0, dx2coul = 0, rmins_coul2 = 0;   // charges: cut-off^2, table spacing, table start^2
  std::vector<int4> krows;   // k rows {ka, kb, kc0, len} of the system's k set
  std::vector<int> krow_k0;  // first k of each row (system-local)
  std::vector<int> ka, kb, kc;
};

// Intramolecular terms beyond bonds and bends, in groups (CM3D's order
// inside a group): cross bonds join level 2 (fbondx md_fbocross.c:40),
// torsions and 1-4 pairs make the torsion level (ftors md_ftors.c:117, fonfo
// md_fonefour.c:70).  1-4 types are numbered across the systems of a batch,
// each with its own table of o14_ntab[t] knots from o14_tab0[t].
struct IntraDev {
  const int *bx_off = nullptr;          // ngroups + 1
  const int4 *bx_ijk = nullptr;         // {i, j, k, -}
  const double4 *bx_par = nullptr;      // {eq1, eq2, fk, -}
  const int *tor_off = nullptr;         // ngroups + 1
  const int4 *tor_ijkl = nullptr;
  const int2 *tor_par = nullptr;        // {form (0 harmonic, 1 cosine series), row}
  const double2 *tor_h = nullptr;       // harmonic rows {eq, fk}
  const double *tor_v = nullptr;        // series rows of CM3D_NB_MAXPOWER_TORS coefficients
  const int *o14_off = nullptr;         // ngroups + 1
  const int4 *o14_ij = nullptr;         // {i, j, type, -}
  const double4 *o14_rng = nullptr;     // per type {rmin2, rmax2, dx2tab, scale}
  const double *o14_se = nullptr;       // per type scale_onefour_e
  const int2 *o14_tab = nullptr;        // per type {first knot, knots}
  const double *o14_v = nullptr, *o14_dv = nullptr;
  const unsigned char *frz = nullptr;   // per atom: frozen (nullptr: none)
};

struct Ctx {
  // ---- configuration
  int dev = 0;
  // ---- systems (a single system is a batch of one)
  int nsys = 1;
  std::vector<SysP> h_sp;              // per-system parameters, host copy
  std::vector<SysH> hs;
  SysP *sp = nullptr;                  // device copy
  int *sys_of = nullptr;               // per atom: its system
  int *cell_sys = nullptr;             // per cell: its system
  int *sreb = nullptr;                 // per system: rebuild requested (nrefsh)
  int *slast = nullptr;                // per system: md_finter.c's isteplast
  long long *sstat = nullptr;          // per system: SS_* counters
  long long *h_sstat = nullptr;
  int *ktile_sys = nullptr, *ftile_sys = nullptr, *k_sys = nullptr;   // k-space tiles / k -> system
  int ktiles_tot = 0, ftiles_tot = 0, nrows_max = 0;
  int ncoul = 0;                       // erfc tables (one per system with charges)
  int all_rebuild = 1;                 // list kernels: rebuild every system (host-driven builds)
  int num_sms = 148;
  size_t smem_optin = 0;               // opt-in shared memory per block (bytes)
  double *ered = nullptr;              // k_ereduce: per-block partial sums of one large system
  unsigned *ered_done = nullptr;       // k_ereduce: blocks finished per quantity
  int lw_cap = 0;                      // staged list build: neighbourhood atoms per block (0: off)
  int *grp_work = nullptr;             // groups with ecorr pairs, bonds or bends (device)
  int ngwork = 0;
  int *rb_scan = nullptr;              // staged list build: cells rebuilt before each system (nsys + 1)
  size_t lw_smem_max = 0;              // its shared-memory limit (bytes)
  int win_ok = 1;                      // single systems may use the windowed pair kernel
  int win_env_off = 0;                 // CM3D_NB_PAIR_KERNEL=list: never
  int pair_used = 0;                   // kernel of the last pair launch (CM3D_NB_PAIR_*)
  int4 *sys_items = nullptr;           // batch pair kernel work items {system, first, end, -}
  int nsys_items = 0;
  float4 *ftab_lj2 = nullptr;          // LJ force + energy coefficients, 2 float4 per knot
  // compact-window pair path (nb_cwin.cu): one system, >= 3 cells per axis
  int cw_ok = 0;                       // set up and valid for this context
  int cw_use = 0;                      // preferred over the window/gather kernels (autotuner)
  int cw_cap = 0;                      // window slots (of the kernel in use)
  int cw_row = 32;                     // compact-list lanes per atom: 32 (k_pair_cw) or 8 (k_pair_cs)
  int cw_cap32 = 0, cw_cap8 = 0;       // window slots of each kernel (k_pair_cs: per block group)
  size_t cw_smem = 0;                  // dynamic shared memory of k_pair_cw
  int cw_words = 0;                    // 8-byte words per atom slot of the compact list
  uint2 *cwl = nullptr;                // compact list (16-bit window indices, lane-interleaved blocks)
  int2 *cwn = nullptr;                 // per sorted atom: LJ-segment and electrostatics-only lengths
  float4 *cw_tf = nullptr;             // erfc force coefficients + base energy
  float2 *cw_tg = nullptr;             // erfc energy slope and curvature
  float4 *cw_tl = nullptr;             // LJ, 2 float4 per knot
  float cw_lj1[4] = {0, 0, 0, 0};      // the one LJ interaction: rc^2, dx2tab, offset, vt
  int cw_nsplit = 1, cw_nitems = 0;    // work items: cells x parts
  int cw_nt = 512;                     // threads per pair-kernel block (512 or 640; autotuner)
  double *cw_part = nullptr;           // per-item FP64 energy/virial sums
  // a batch: the systems with >= 3 cells per axis in the compact kernel (in
  // groups of systems with the same tables), the others in the gather kernel
  int cw_batch = 0;
  int *cw_sys = nullptr;               // per system: 1 = compact (device)
  int2 *cw_sitems = nullptr;           // per system: its items {first, count} (device)
  int4 *cw_items = nullptr;            // {system, cell of the system, part, parts}, by group (device)
  int *cw_gidx = nullptr;              // sorted atoms of the gather-kernel systems (device)
  int *cw_scan = nullptr;              // atoms to convert before each system (nsys + 1, device)
  int cw_ng = 0;
  void *cw_grp = nullptr;              // the groups (host, nb_cwin.cu)
  const int *pair_gidx = nullptr;      // a gather launch over these sorted atoms only
  int pair_ng = 0;
  int stage_ntypes = 0, stage_ninter = 0;   // largest per-system type count / interaction count
  cudaStream_t st = nullptr;
  cudaStream_t st2 = nullptr;                // side stream: force(1)'s k-space beside the list build
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // registered page-locked host outputs (cm3d_nb_set_host_outputs): every
  // step copies its final positions (on st3, beside the rest of the step)
  // and velocities there
  double *ho_pos = nullptr, *ho_vel = nullptr;
  cudaStream_t st3 = nullptr;
  cudaEvent_t ev_f3 = nullptr, ev_j3 = nullptr;
  bool ho_forked = false;
  int mode = CM3D_NB_MIXED;
  int need_short = 0;
  int tpa = 0;
  double cell_scale = 1.0;   // list cells at least this many list radii wide
  int use_graph = 1;
  // ---- sizes and scalars
  int n = 0, ntypes = 0, ninter = 0, ntable = 0, ncharge = 0, ktot = 0, necorr = 0;
  int nbonds = 0, nbends = 0, nres_lrf = 1, nres_intra = 1, nres_tors = 1, ndof = 1;
  int iperd = 3;
  double dt = 0, vlrc = 0, wlrc = 0, skin = 0, rheal = 0;
  double hmat[9], hmati[9];
  double rlist_max = 0;        // largest list radius (LJ or charge, with skin)
  double rc_lj_max = 0;
  double kappa = 0, kappa2 = 0, falp2 = 0, ewald_self = 0, ewald_bkg = 0;
  double dx2coul = 0, rmins_coul2 = 0, rmaxs_coul2 = 0, rminl_coul2 = 0, rmaxl_coul2 = 0;
  double rmaxs_skin2_e = 0, rmaxl_skin2_e = 0;
  double tablast_e = 0;        // coultab[ntable-4] (finter_e.c:67)
  // ---- per-atom device arrays (original order)
  double *pos = nullptr, *vel = nullptr, *fxl = nullptr, *fxs = nullptr, *fxa = nullptr;
  double *fxr = nullptr;                // torsion level (torsions + 1-4 pairs)
  double *mass = nullptr, *q = nullptr, *dxn = nullptr, *snap = nullptr;
  int *itype = nullptr;
  // ---- parameters on device
  int *map = nullptr;                   // ntypes^2
  double *vtab = nullptr, *dvtab = nullptr, *switchs = nullptr;   // ninter*ntable
  double *icut = nullptr;               // 8*ninter: rmaxs_cut2 rmins_cut2 rmaxl_cut2
                                        // rminl_cut2 rmaxs_skin2 rmaxl_skin2 dx2tab vt[ntm4]
  double *coultab = nullptr, *dcoultab = nullptr, *switchse = nullptr;
  int *excl_off = nullptr, *excl_idx = nullptr, *cexcl_off = nullptr, *cexcl_idx = nullptr;
  // FP32 coefficient tables (mixed): per index k two float4
  //   LJ:   {dv0, dvA, dvB, v0} {vA, vB, sw0, swA}  + swB in a third
  //   elec: {dc0, dcA, dcB, c0} {cA, cB, 0, 0}
  float4 *ftab_lj = nullptr;            // 3 * ninter * ntable
  float4 *ftab_el = nullptr;            // 2 * ntable
  float *fcut = nullptr;                // 6*ninter FP32: rmaxl_cut2 rmins*dx2 dx2 rminl_cut2 rmaxs_cut2 vt[ntm4]
  // ---- Ewald
  int nrows = 0;                        // k rows of constant (ka, kb)
  int4 *rows = nullptr;                 // {ka, kb, kc_lo, len}
  int *row_k0 = nullptr;                // index of the row's first k
  double2 *sk = nullptr;                // S(k) FP64
  double2 *spart = nullptr;             // per-tile partial S(k)
  float2 *akf = nullptr;                // 2 preg S(k), FP32 (mixed)
  double2 *akd = nullptr;               // 2 preg S(k), FP64 (plain)
  uint4 *kfrac = nullptr;               // per charged atom: fixed-point fractional coords + tq
  double4 *kposd = nullptr;             // per charged atom (plain): x y z tq
  int *icharge = nullptr;
  int *ka_d = nullptr, *kb_d = nullptr, *kc_d = nullptr;
  int ks_tiles = 0, ks_tile_atoms = 0, kf_split = 1;
  bool ks_small = false;                // batch of systems with <= 32 charges: one-warp k-space tiles
  size_t kf_smem = 0;
  double *kf_part = nullptr;            // per row split partial reciprocal forces (mixed, split > 1)
  int2 *ecorr_pairs = nullptr;          // CM3D's iecorr/jecorr order
  // ---- bonded groups (connected components of bonds/bends/ecorr)
  int ngroups = 0;
  int *grp_atom_off = nullptr, *grp_atoms = nullptr;
  int *grp_bond_off = nullptr, *grp_bend_off = nullptr, *grp_ecorr_off = nullptr;
  int4 *bond_ij = nullptr;              // {i, j, -, -} grouped order
  double2 *bond_p = nullptr;            // {eq, fk}
  int4 *bend_ijk = nullptr;
  double2 *bend_p = nullptr;
  int2 *ecorr_ij = nullptr;             // grouped order
  IntraDev intra;                       // cross bonds, torsions, 1-4 pairs, frozen atoms
  bool has_tors_level = false;          // any torsion or 1-4 pair
  bool has_intra_x = false;             // any cross bond, torsion or 1-4 pair
  double *intra_buf = nullptr;          // one allocation behind the IntraDev arrays
  // Nose-Hoover chains (NVT): thermostats numbered across the batch's systems
  int ntherm = 0, nchain = 0;
  int *ithm = nullptr;                  // per atom: its thermostat, -1 none
  double *nhc = nullptr;                // mnh | gkt | eta | veta | feta, ntherm * nchain each, then p2m (ntherm)
  std::vector<int> therm0;              // per system: its first thermostat (nsys + 1 entries)
  // kinetic sums of the thermostats in a fixed order: per-atom terms m v^2
  // (nvt_kin), summed by one warp per chunk of at most NVT_CHUNK atoms of one
  // thermostat (th_atoms in thermostat order, th_chunk {first, end}), the
  // chunks of thermostat j (th_choff[j] .. th_choff[j + 1]) added in order
  double *nvt_kin = nullptr, *nvt_chsum = nullptr;
  int *th_atoms = nullptr, *th_choff = nullptr;
  int2 *th_chunk = nullptr;
  int nth_chunks = 0;
  // ---- cell grid and lists
  int nc[3] = {1, 1, 1}, ncells = 1;
  int *cell_of = nullptr, *cell_start = nullptr, *cell_cursor = nullptr, *cell_atoms = nullptr;
  int *rank = nullptr;                  // original -> sorted
  int *cnt = nullptr;                   // 5 per atom counts (t s te se full)
  long long *off = nullptr;             // 5*(n+1) exclusive offsets
  long long *ltot = nullptr;            // LT_COUNT device totals
  long long lcap[LT_COUNT] = {0, 0, 0, 0, 0};
  long long hcount[LT_COUNT] = {0, 0, 0, 0, 0};
  int2 *lst[4] = {nullptr, nullptr, nullptr, nullptr};   // t s te se half lists
  uint32_t *nbr = nullptr;              // full list (mixed): n slots of nbr_stride entries
  int *nlen = nullptr;                  // full-list length per sorted atom
  int nbr_stride = 0;
  float4 *xq = nullptr;                 // sorted: cell-relative FP32 pos + q
  float *epart = nullptr;               // mixed: per-atom energy/virial partials
  int *styp = nullptr;                  // sorted type
  int *sorig = nullptr;                 // sorted -> original (== cell_atoms)
  float4 *shift = nullptr;              // 27 FP32 cell-shift vectors
  double *corner = nullptr;             // per sorted atom cell-origin offset (3n FP64)
  int4 *cimg = nullptr;                 // per atom: packed cell coords | periodic image
  // ---- accumulators, status, state
  double *acc = nullptr;
  long long *stat = nullptr;
  int *istate = nullptr;
  double *h_acc = nullptr;              // pinned mirrors
  long long *h_stat = nullptr;
  int *h_istate = nullptr;
  long long *h_ltot = nullptr;
  // ---- host bookkeeping
  bool lists_built = false;
  bool forces_valid = false;
  bool want_half = false;               // mixed mode: also write the half lists
  bool no_snapshot = false;             // a rebuild that must not touch dxn
  long long launches = 0;
  long long rebuilds_host = 0, overflows_host = 0;
  Timing timing;
  cudaGraphExec_t graph = nullptr;
  long long graph_launches = 0;
  const int *gate = nullptr;            // istate while a step is being captured
  cudaEvent_t step_ev = nullptr;        // end of asynchronously launched steps
  bool pending = false;                 // steps launched and not finished yet
  int pend_istep0 = 0, pend_nsteps = 0;
  std::string name;
};

// ------------------------------------------------------------ error handling
void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);
#define CK(call)                                        \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)
#define CKL(ctx) CK(cudaPeekAtLastError())

// timing helpers (class: 0 pair, 1 kspace, 2 list, 3 integrate)
void tbegin(Ctx *c, int cls, cudaEvent_t *e0);
void tend(Ctx *c, int cls, cudaEvent_t e0);

// ------------------------------------------------------------ device helpers
// anint of CM3D's Linux build (include/md_macros.h:52): truncation toward
// zero of A +/- 0.5, i.e. round half away from zero
__device__ __forceinline__ double anint_ref(double a) {
  return (double)(int)(a >= 0.0 ? __dadd_rn(a, 0.5) : __dadd_rn(a, -0.5));
}

// period_new (integrate/md_period.new.c:39-52) for one displacement, in
// CM3D's operation order with every product and sum rounded separately (no
// FMA contraction) so that r^2 is bit-identical to CM3D's
__device__ __forceinline__ void period_ref(double &dx, double &dy, double &dz,
                                           const double *h, const double *hi) {
  double sx = __dadd_rn(__dadd_rn(__dmul_rn(dx, hi[0]), __dmul_rn(dy, hi[1])), __dmul_rn(dz, hi[2]));
  double sy = __dadd_rn(__dadd_rn(__dmul_rn(dx, hi[3]), __dmul_rn(dy, hi[4])), __dmul_rn(dz, hi[5]));
  double sz = __dadd_rn(__dadd_rn(__dmul_rn(dx, hi[6]), __dmul_rn(dy, hi[7])), __dmul_rn(dz, hi[8]));
  sx = __dsub_rn(sx, anint_ref(sx));
  sy = __dsub_rn(sy, anint_ref(sy));
  sz = __dsub_rn(sz, anint_ref(sz));
  dx = __dadd_rn(__dadd_rn(__dmul_rn(sx, h[0]), __dmul_rn(sy, h[1])), __dmul_rn(sz, h[2]));
  dy = __dadd_rn(__dadd_rn(__dmul_rn(sx, h[3]), __dmul_rn(sy, h[4])), __dmul_rn(sz, h[5]));
  dz = __dadd_rn(__dadd_rn(__dmul_rn(sx, h[6]), __dmul_rn(sy, h[7])), __dmul_rn(sz, h[8]));
}

__device__ __forceinline__ double r2_ref(double dx, double dy, double dz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// membership of (i, j) in a CSR exclusion list stored at the lower index
__device__ __forceinline__ bool excluded(int i, int j, const int *__restrict__ off,
                                         const int *__restrict__ idx) {
  int a = i < j ? i : j, b = i < j ? j : i;
  int lo = off[a], hi = off[a + 1];
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    int v = idx[mid];
    if (v == b) return true;
    if (v < b) lo = mid + 1;
    else hi = mid;
  }
  return false;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block-wide sum of NV doubles into acc[slot..slot+NV) with one atomic per
// value per block; all threads of the block must call it
template <int NV>
__device__ __forceinline__ void block_acc(double (&v)[NV], double *acc, const int *slots) {
  __shared__ double red[32][NV];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) red[w][k] = v[k];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double s = lane < nw ? red[lane][k] : 0.0;
      s = warp_sum(s);
      if (lane == 0 && s != 0.0) atomicAdd(acc + slots[k], s);
    }
  }
}

// ------------------------------------------------------------ host helpers
int plain_pairs(Ctx *c, int iflg, int which);   // nb_plain.cu
int plain_ecorr(Ctx *c, const int2 *ij);        // nb_plain.cu
int mixed_pairs(Ctx *c, int iflg, int mask);    // nb_pair.cu
bool win_applies(Ctx *c);                       // nb_pair.cu: windowed pair kernel possible
int build_lists(Ctx *c, bool device_flag, bool all);   // nb_list.cu
// Held across every CUDA call that can synchronize the whole device (context
// creation and destruction, allocation and freeing at run time) and across
// every graph capture: a device-wide synchronization from one host thread
// while another captures a step graph would invalidate that capture.
std::recursive_mutex &device_mutex();           // nb_capi.cu
using DevLock = std::lock_guard<std::recursive_mutex>;
int list_setup(Ctx *c);                         // nb_list.cu
void cell_shifts(SysP &P, const SysH &H);       // nb_list.cu
int refresh_corners(Ctx *c);                    // nb_list.cu: cell corners under a new box
int pair_forces(Ctx *c, int iflg, int which);   // nb_pair.cu: which 0 LJ, 1 elec, 2 fused
int pair_setup(Ctx *c);                         // nb_pair.cu
int cw_setup(Ctx *c);                           // nb_cwin.cu: compact-window path (after pair_setup)
constexpr int CW_MAX_SPLIT = 8;                 // most parts a cell's atoms are split into
void cw_set_split(Ctx *c, int nsplit);          // nb_cwin.cu
constexpr int CM3D_CW_ROW = 32;                 // compact-list rows (lanes per atom) of k_pair_cw
constexpr int CM3D_CS_LPA = 8;                  //   and of k_pair_cs
constexpr int CM3D_CS_THREADS = 512;            // k_pair_cs block: four groups of four warps
int cw_set_row(Ctx *c, int row);
int host_outputs_tail(Ctx *c);                  // nb_step.cu: end of a step with registered host outputs                // nb_cwin.cu: a batch's list layout, 32 or 8 lanes per atom
int cw_convert(Ctx *c, bool device_flag, bool all);   // nb_cwin.cu: master list -> compact list
void cw_destroy(Ctx *c);                        // nb_cwin.cu: host-side group data
bool cw_applies(Ctx *c, int iflg, bool ns);     // nb_cwin.cu
int cw_pairs(Ctx *c, int mask, double *fout);   // nb_cwin.cu: pair kernel launch
int cw_ereduce(Ctx *c, int mask);               // nb_cwin.cu: its energy/virial sums
int kspace_forces(Ctx *c);                      // nb_kspace.cu
bool kspace_async_ok(const Ctx *c);             // nb_kspace.cu: force(1)'s k-space beside the lists/pairs
int kspace_fork(Ctx *c);                        // nb_kspace.cu
int kspace_join(Ctx *c);                        // nb_kspace.cu
int kspace_setup(Ctx *c);                       // nb_kspace.cu
int step_setup(Ctx *c, const cm3d_nb_system *systems, int nsys);   // nb_step.cu
int run_step(Ctx *c, int istep0, int nsteps);   // nb_step.cu
int launch_steps(Ctx *c, int istep0, int nsteps);   // nb_step.cu
int finish_steps(Ctx *c);                       // nb_step.cu
int query_steps(Ctx *c, int *done);             // nb_step.cu
int run_force(Ctx *c, int iflg);                // nb_step.cu
int run_bonded(Ctx *c);                         // nb_step.cu
int group_init(Ctx *c, bool zero_fxs);          // nb_step.cu
int finish_level1(Ctx *c, double dter, double dter1, bool kick);   // nb_step.cu
int check_displacement(Ctx *c);                 // nb_step.cu
int reset_positions(Ctx *c);                    // nb_step.cu

inline int grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 2147483647LL) g = 2147483647LL;
  return (int)g;
}

}  // namespace cm3d
