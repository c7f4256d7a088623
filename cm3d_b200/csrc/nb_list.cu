// nb_list.cu -- link-cell binning and Verlet-list build on the GPU.
//
// Replaces get_ngbr (energy/control/ngbr_list.c:297-581), ngbr_list
// (ngbr_list.c:35-101), get_ngbr_e (energy/control/elec_ngbr.c:220-358),
// ngbr_liste (ngbr_list.c:103-143) and the link-cell helpers get_lnklist /
// get_lnklist_e (energy/control/set_link.c:203-300).
//
// Pair membership is decided exactly as CM3D decides it: the displacement is
// taken in FP64, folded with period_ref() (md_period.new.c:39-52, CM3D's
// anint and operation order, no FMA contraction -- this file is compiled with
// -fmad=false as well) and compared with the per-interaction radius
// rmaxl_skin2[map[ti][tj]] / rmaxs_skin2 (LJ, after the map == -1 and
// exclusion tests) or rmaxl_skin2_e / rmaxs_skin2_e (charged atoms, after the
// charge-exclusion test).  The resulting pair sets are bit-identical to
// CM3D's.  The cell grid itself is our own: cells at least one list radius
// wide, atoms counting-sorted by cell (order inside a cell by atom index), and
// a stencil of unique neighbour cells, so every pair within range is seen
// exactly once per direction whatever CM3D's ncell_div is.
//
// Outputs
//   lst[0..3]  CM3D's four half lists t, s, te, se as (i, j) with i < j
//   nbr        (mixed mode) a full list per atom in cell-sorted order; each
//              32-bit entry holds j's sorted index, the code of the cell shift
//              that turns cell-relative coordinates into the minimum-image
//              displacement, and whether the pair is in the t and/or te list
//   xq, styp   cell-relative FP32 coordinates + charge and type, sorted order
#include <math.h>
#include <stdio.h>

#include "nb_common.cuh"

namespace cm3d {

// ----------------------------------------------------------------- binning
__global__ void k_cell_assign(int n, const double *__restrict__ pos, const double *__restrict__ hmati,
                              int ncx, int ncy, int ncz, int *__restrict__ cell_of,
                              int *__restrict__ cell_count, int4 *__restrict__ cimg,
                              const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x = pos[i], y = pos[n + i], z = pos[2 * n + i];
  double s[3];
  for (int d = 0; d < 3; d++)
    s[d] = __dadd_rn(__dadd_rn(__dmul_rn(x, hmati[3 * d]), __dmul_rn(y, hmati[3 * d + 1])),
                     __dmul_rn(z, hmati[3 * d + 2]));
  int img[3], cc[3];
  int ncd[3] = {ncx, ncy, ncz};
  for (int d = 0; d < 3; d++) {
    double fl = floor(s[d]);
    double fr = s[d] - fl;                       // [0, 1]
    int c = (int)(fr * ncd[d]);
    c = c < 0 ? 0 : (c >= ncd[d] ? ncd[d] - 1 : c);
    img[d] = (int)fl;
    cc[d] = c;
  }
  int cell = (cc[0] * ncy + cc[1]) * ncz + cc[2];
  cell_of[i] = cell;
  cimg[i] = make_int4(cc[0] | (cc[1] << 10) | (cc[2] << 20), img[0], img[1], img[2]);
  atomicAdd(cell_count + cell, 1);
}

// exclusive scan of `m` ints (or long longs) in one block; `nseg` independent
// segments laid out back to back, one per blockIdx.y; segment totals go to
// tot[blockIdx.y]
template <typename TI, typename TO>
__global__ void k_scan(const TI *__restrict__ in, TO *__restrict__ out, long long *__restrict__ tot,
                       int m, const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  const TI *a = in + (size_t)blockIdx.y * m;
  TO *o = out + (size_t)blockIdx.y * (m + 1);
  __shared__ TO part[1024];
  int t = threadIdx.x, nt = blockDim.x;
  int chunk = (m + nt - 1) / nt;
  int lo = t * chunk, hi = min(m, lo + chunk);
  TO s = 0;
  for (int k = lo; k < hi; k++) s += (TO)a[k];
  part[t] = s;
  __syncthreads();
  for (int d = 1; d < nt; d <<= 1) {
    TO v = t >= d ? part[t - d] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  TO run = t > 0 ? part[t - 1] : 0;
  for (int k = lo; k < hi; k++) {
    o[k] = run;
    run += (TO)a[k];
  }
  if (t == nt - 1) {
    o[m] = part[nt - 1];
    if (tot) tot[blockIdx.y] = (long long)part[nt - 1];
  }
}

__global__ void k_cell_fill(int n, const int *__restrict__ cell_of, const int *__restrict__ cell_start,
                            int *__restrict__ cursor, int *__restrict__ cell_atoms,
                            const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = cell_of[i];
  int slot = atomicAdd(cursor + c, 1);
  cell_atoms[cell_start[c] + slot] = i;
}

// order every cell's atoms by atom index (deterministic lists)
__global__ void k_cell_sort(int ncells, const int *__restrict__ cell_start, int *__restrict__ cell_atoms,
                            const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  int lo = cell_start[c], hi = cell_start[c + 1];
  for (int a = lo + 1; a < hi; a++) {
    int v = cell_atoms[a], b = a - 1;
    while (b >= lo && cell_atoms[b] > v) {
      cell_atoms[b + 1] = cell_atoms[b];
      b--;
    }
    cell_atoms[b + 1] = v;
  }
}

struct ListParams {
  int n, ntypes, ncx, ncy, ncz;
  int sx[3], sy[3], sz[3];          // unique stencil offsets per dimension
  int nsx, nsy, nsz;
  double h[9], hi[9];
  double rmaxl_skin2_e, rmaxs_skin2_e;
  int want_full;                    // mixed: build the full list too
  long long cap[LT_COUNT];
};

// Visit every candidate j of sorted atom t, call f(i, j, flags, code) for
// each pair that belongs to at least one list.  flags: bit0 t, bit1 s,
// bit2 te, bit3 se.  code: cell-shift code for the full list.
template <typename F>
__device__ __forceinline__ void for_pairs(const ListParams &P, int t, const int *__restrict__ cell_atoms,
                                          const int *__restrict__ cell_start, const double *__restrict__ pos,
                                          const int *__restrict__ itype, const int *__restrict__ map,
                                          const double *__restrict__ icut, const double *__restrict__ q,
                                          const int *__restrict__ excl_off, const int *__restrict__ excl_idx,
                                          const int *__restrict__ cexcl_off, const int *__restrict__ cexcl_idx,
                                          const int4 *__restrict__ cimg, int ninter, F f) {
  const int n = P.n;
  int i = cell_atoms[t];
  int4 ci = cimg[i];
  int cx = ci.x & 1023, cy = (ci.x >> 10) & 1023, cz = (ci.x >> 20) & 1023;
  double xi = pos[i], yi = pos[n + i], zi = pos[2 * n + i];
  int ti = itype[i];
  bool qi = q[i] != 0.0;
  for (int a = 0; a < P.nsx; a++) {
    int jx = cx + P.sx[a];
    jx = jx < 0 ? jx + P.ncx : (jx >= P.ncx ? jx - P.ncx : jx);
    for (int b = 0; b < P.nsy; b++) {
      int jy = cy + P.sy[b];
      jy = jy < 0 ? jy + P.ncy : (jy >= P.ncy ? jy - P.ncy : jy);
      for (int cc = 0; cc < P.nsz; cc++) {
        int jz = cz + P.sz[cc];
        jz = jz < 0 ? jz + P.ncz : (jz >= P.ncz ? jz - P.ncz : jz);
        int cell = (jx * P.ncy + jy) * P.ncz + jz;
        int lo = cell_start[cell], hi = cell_start[cell + 1];
        for (int u = lo; u < hi; u++) {
          int j = cell_atoms[u];
          if (j == i) continue;
          if (!P.want_full && j < i) continue;
          int intr = map[ti * P.ntypes + itype[j]];
          bool qj = q[j] != 0.0;
          bool lj_ok = intr >= 0;
          bool el_ok = qi && qj;
          if (!lj_ok && !el_ok) continue;
          double dx = xi - pos[j], dy = yi - pos[n + j], dz = zi - pos[2 * n + j];
          // image of CM3D's min image (needed for the shift code)
          double sx = __dadd_rn(__dadd_rn(__dmul_rn(dx, P.hi[0]), __dmul_rn(dy, P.hi[1])), __dmul_rn(dz, P.hi[2]));
          double sy = __dadd_rn(__dadd_rn(__dmul_rn(dx, P.hi[3]), __dmul_rn(dy, P.hi[4])), __dmul_rn(dz, P.hi[5]));
          double sz = __dadd_rn(__dadd_rn(__dmul_rn(dx, P.hi[6]), __dmul_rn(dy, P.hi[7])), __dmul_rn(dz, P.hi[8]));
          double mx = anint_ref(sx), my = anint_ref(sy), mz = anint_ref(sz);
          sx = __dsub_rn(sx, mx);
          sy = __dsub_rn(sy, my);
          sz = __dsub_rn(sz, mz);
          double ex = __dadd_rn(__dadd_rn(__dmul_rn(sx, P.h[0]), __dmul_rn(sy, P.h[1])), __dmul_rn(sz, P.h[2]));
          double ey = __dadd_rn(__dadd_rn(__dmul_rn(sx, P.h[3]), __dmul_rn(sy, P.h[4])), __dmul_rn(sz, P.h[5]));
          double ez = __dadd_rn(__dadd_rn(__dmul_rn(sx, P.h[6]), __dmul_rn(sy, P.h[7])), __dmul_rn(sz, P.h[8]));
          double r2 = r2_ref(ex, ey, ez);
          int flags = 0;
          if (lj_ok) {
            if (r2 < icut[8 * intr + 5] && !excluded(i, j, excl_off, excl_idx)) {
              flags |= 1;
              if (r2 < icut[8 * intr + 4]) flags |= 2;
            }
          }
          if (el_ok) {
            if (r2 < P.rmaxl_skin2_e && !excluded(i, j, cexcl_off, cexcl_idx)) {
              flags |= 4;
              if (r2 < P.rmaxs_skin2_e) flags |= 8;
            }
          }
          if (!flags) continue;
          int4 cj = cimg[j];
          int kx = (ci.y - cj.y - (int)mx) * P.ncx + (cx - (cj.x & 1023));
          int ky = (ci.z - cj.z - (int)my) * P.ncy + (cy - ((cj.x >> 10) & 1023));
          int kz = (ci.w - cj.w - (int)mz) * P.ncz + (cz - ((cj.x >> 20) & 1023));
          // |k| <= 1 per dimension whenever r < rlist <= cell width; any
          // other value would mean the geometry assumption broke: count it
          // and use the zero shift rather than index past the shift table
          int code = (kx + 1) * 9 + (ky + 1) * 3 + (kz + 1);
          if (kx < -1 || kx > 1 || ky < -1 || ky > 1 || kz < -1 || kz > 1) {
            code = 13;
            flags |= 16;
          }
          f(i, j, flags, code);
        }
      }
    }
  }
}

__global__ void k_list_count(ListParams P, const int *__restrict__ cell_atoms, const int *__restrict__ cell_start,
                             const double *__restrict__ pos, const int *__restrict__ itype,
                             const int *__restrict__ map, const double *__restrict__ icut,
                             const double *__restrict__ q, const int *__restrict__ excl_off,
                             const int *__restrict__ excl_idx, const int *__restrict__ cexcl_off,
                             const int *__restrict__ cexcl_idx, const int4 *__restrict__ cimg, int ninter,
                             int *__restrict__ cnt, const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.n) return;
  int c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0;
  for_pairs(P, t, cell_atoms, cell_start, pos, itype, map, icut, q, excl_off, excl_idx, cexcl_off,
            cexcl_idx, cimg, ninter, [&](int i, int j, int fl, int) {
              if (j > i) {
                c0 += fl & 1;
                c1 += (fl >> 1) & 1;
                c2 += (fl >> 2) & 1;
                c3 += (fl >> 3) & 1;
              }
              if (fl & 5) c4++;
            });
  cnt[t] = c0;
  cnt[P.n + t] = c1;
  cnt[2 * P.n + t] = c2;
  cnt[3 * P.n + t] = c3;
  cnt[4 * P.n + t] = P.want_full ? c4 : 0;
}

__global__ void k_list_fill(ListParams P, const int *__restrict__ cell_atoms, const int *__restrict__ cell_start,
                            const double *__restrict__ pos, const int *__restrict__ itype,
                            const int *__restrict__ map, const double *__restrict__ icut,
                            const double *__restrict__ q, const int *__restrict__ excl_off,
                            const int *__restrict__ excl_idx, const int *__restrict__ cexcl_off,
                            const int *__restrict__ cexcl_idx, const int4 *__restrict__ cimg, int ninter,
                            const long long *__restrict__ off, const long long *__restrict__ tot,
                            const int *__restrict__ rank, int2 *__restrict__ l0, int2 *__restrict__ l1,
                            int2 *__restrict__ l2, int2 *__restrict__ l3, uint32_t *__restrict__ nbr,
                            long long *__restrict__ stat, int *__restrict__ halt,
                            const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.n) return;
  // if any list outgrew its capacity nothing is written and the step halts:
  // the host grows the buffers and finishes the step (see run_step)
  bool ok0 = tot[0] <= P.cap[0], ok1 = tot[1] <= P.cap[1], ok2 = tot[2] <= P.cap[2],
       ok3 = tot[3] <= P.cap[3], ok4 = tot[4] <= P.cap[4];
  if (!(ok0 && ok1 && ok2 && ok3 && ok4)) {
    if (t == 0) {
      atomicAdd((unsigned long long *)(stat + ST_OVERFLOW), 1ull);
      if (halt) *halt = 1;
    }
    return;
  }
  long long p0 = off[t], p1 = off[(P.n + 1) + t], p2 = off[2 * (P.n + 1) + t],
            p3 = off[3 * (P.n + 1) + t], p4 = off[4 * (P.n + 1) + t];
  for_pairs(P, t, cell_atoms, cell_start, pos, itype, map, icut, q, excl_off, excl_idx, cexcl_off,
            cexcl_idx, cimg, ninter, [&](int i, int j, int fl, int code) {
              if (j > i) {
                int2 pr = make_int2(i, j);
                if ((fl & 1) && ok0) l0[p0++] = pr;
                if ((fl & 2) && ok1) l1[p1++] = pr;
                if ((fl & 4) && ok2) l2[p2++] = pr;
                if ((fl & 8) && ok3) l3[p3++] = pr;
              }
              if (fl & 16) atomicAdd((unsigned long long *)(stat + ST_BADSHIFT), 1ull);
              if (P.want_full && (fl & 5) && ok4) {
                uint32_t e = (uint32_t)rank[j] | ((uint32_t)code << ENT_CODE_SHIFT);
                if (fl & 1) e |= ENT_LJ;
                if (fl & 2) e |= ENT_LJS;
                if (fl & 4) e |= ENT_EL;
                if (fl & 8) e |= ENT_ELS;
                nbr[p4++] = e;
              }
            });
}

// sorted-order arrays of the mixed engine: rank, type, FP64 cell corner
// (the cell origin in Cartesian coordinates, held fixed until the next
// rebuild) and the first FP32 cell-relative coordinates
__global__ void k_sorted_init(int n, const int *__restrict__ cell_atoms, const int4 *__restrict__ cimg,
                              const double *__restrict__ h, int ncx, int ncy, int ncz,
                              const int *__restrict__ itype, int *__restrict__ rank,
                              int *__restrict__ styp, double *__restrict__ corner,
                              const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int i = cell_atoms[t];
  int4 ci = cimg[i];
  double o0 = (double)ci.y + (double)(ci.x & 1023) / ncx;
  double o1 = (double)ci.z + (double)((ci.x >> 10) & 1023) / ncy;
  double o2 = (double)ci.w + (double)((ci.x >> 20) & 1023) / ncz;
  corner[t] = h[0] * o0 + h[1] * o1 + h[2] * o2;
  corner[n + t] = h[3] * o0 + h[4] * o1 + h[5] * o2;
  corner[2 * n + t] = h[6] * o0 + h[7] * o1 + h[8] * o2;
  rank[i] = t;
  styp[t] = itype[i];
}

__global__ void k_snapshot(int n3, const double *__restrict__ pos, double *__restrict__ dxn,
                           const int *__restrict__ gate, int *__restrict__ istate,
                           long long *__restrict__ stat) {
  if (gated_off(gate, 1)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) dxn[i] = pos[i];
  if (i == 0) {
    // md_finter.c:98: isteplast = istep after a rebuild
    istate[IS_ISTEPLAST] = istate[IS_ISTEP];
    atomicAdd((unsigned long long *)(stat + ST_REBUILDS), 1ull);
  }
}

// --------------------------------------------------------------- host side
static void stencil(int nc, int *s, int *ns) {
  if (nc >= 3) {
    s[0] = -1; s[1] = 0; s[2] = 1; *ns = 3;
  } else if (nc == 2) {
    s[0] = 0; s[1] = 1; *ns = 2;
  } else {
    s[0] = 0; *ns = 1;
  }
}

int list_setup(Ctx *c) {
  // cells at least one list radius wide in every fractional direction
  // (plane spacing 1/|row d of hmati|)
  int tot = 1;
  for (int d = 0; d < 3; d++) {
    double w = 1.0 / sqrt(c->hmati[3 * d] * c->hmati[3 * d] + c->hmati[3 * d + 1] * c->hmati[3 * d + 1] +
                          c->hmati[3 * d + 2] * c->hmati[3 * d + 2]);
    int m = c->rlist_max > 0 ? (int)floor(w / c->rlist_max) : 1;
    m = m < 1 ? 1 : (m > 1000 ? 1000 : m);
    c->nc[d] = m;
    tot *= m;
  }
  c->ncells = tot;
  CK(cudaMalloc(&c->cell_of, sizeof(int) * (size_t)c->n));
  CK(cudaMalloc(&c->cell_start, sizeof(int) * ((size_t)tot + 1)));
  CK(cudaMalloc(&c->cell_cursor, sizeof(int) * ((size_t)tot + 1)));
  CK(cudaMalloc(&c->cell_atoms, sizeof(int) * (size_t)c->n));
  CK(cudaMalloc(&c->rank, sizeof(int) * (size_t)c->n));
  CK(cudaMalloc(&c->cnt, sizeof(int) * 5 * (size_t)c->n));
  CK(cudaMalloc(&c->off, sizeof(long long) * 5 * ((size_t)c->n + 1)));
  CK(cudaMalloc(&c->ltot, sizeof(long long) * LT_COUNT));
  CK(cudaMallocHost(&c->h_ltot, sizeof(long long) * LT_COUNT));
  CK(cudaMalloc(&c->styp, sizeof(int) * (size_t)c->n));
  CK(cudaMalloc(&c->corner, sizeof(double) * 3 * (size_t)c->n));
  CK(cudaMalloc(&c->xq, sizeof(float4) * (size_t)c->n));
  CK(cudaMalloc(&c->cimg, sizeof(int4) * (size_t)c->n));
  return CM3D_NB_OK;
}

// grow list buffers to hold at least `need` entries (with 30% headroom)
static int grow(Ctx *c, int which, long long need) {
  if (need <= c->lcap[which]) return CM3D_NB_OK;
  long long cap = need + need / 3 + 1024;
  if (which < 4) {
    if (c->lst[which]) cudaFree(c->lst[which]);
    c->lst[which] = nullptr;
    cudaError_t e = cudaMalloc(&c->lst[which], sizeof(int2) * (size_t)cap);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(list)");
  } else {
    if (c->nbr) cudaFree(c->nbr);
    c->nbr = nullptr;
    cudaError_t e = cudaMalloc(&c->nbr, sizeof(uint32_t) * (size_t)cap);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(full list)");
  }
  c->lcap[which] = cap;
  return CM3D_NB_OK;
}

static ListParams params(Ctx *c) {
  ListParams P;
  P.n = c->n;
  P.ntypes = c->ntypes;
  P.ncx = c->nc[0];
  P.ncy = c->nc[1];
  P.ncz = c->nc[2];
  stencil(c->nc[0], P.sx, &P.nsx);
  stencil(c->nc[1], P.sy, &P.nsy);
  stencil(c->nc[2], P.sz, &P.nsz);
  for (int k = 0; k < 9; k++) {
    P.h[k] = c->hmat[k];
    P.hi[k] = c->hmati[k];
  }
  P.rmaxl_skin2_e = c->ncharge > 0 ? c->rmaxl_skin2_e : -1.0;
  P.rmaxs_skin2_e = c->ncharge > 0 ? c->rmaxs_skin2_e : -1.0;
  P.want_full = c->mode == CM3D_NB_MIXED;
  for (int k = 0; k < LT_COUNT; k++) P.cap[k] = c->lcap[k];
  return P;
}

// Build all lists.  With device_flag the kernels are gated on the device
// rebuild flag (for graph replay) and capacity is not re-checked on the host.
int build_lists(Ctx *c, bool device_flag) {
  const int n = c->n;
  const int B = 256;
  const int *gate = device_flag ? c->istate : nullptr;
  cudaEvent_t e0;
  tbegin(c, 2, &e0);
  int4 *cimg = c->cimg;
  CK(cudaMemsetAsync(c->cell_start, 0, sizeof(int) * ((size_t)c->ncells + 1), c->st));
  CK(cudaMemsetAsync(c->cell_cursor, 0, sizeof(int) * ((size_t)c->ncells + 1), c->st));
  double *dhmati = c->acc + ACC_COUNT;        // device copies of hmat/hmati
  double *dhmat = c->acc + ACC_COUNT + 9;
  k_cell_assign<<<grid_for(n, B), B, 0, c->st>>>(n, c->pos, dhmati, c->nc[0], c->nc[1], c->nc[2],
                                                  c->cell_of, c->cell_cursor, cimg, gate);
  k_scan<int, int><<<dim3(1, 1), 1024, 0, c->st>>>(c->cell_cursor, c->cell_start, nullptr, c->ncells, gate);
  CK(cudaMemsetAsync(c->cell_cursor, 0, sizeof(int) * ((size_t)c->ncells + 1), c->st));
  k_cell_fill<<<grid_for(n, B), B, 0, c->st>>>(n, c->cell_of, c->cell_start, c->cell_cursor, c->cell_atoms, gate);
  k_cell_sort<<<grid_for(c->ncells, 128), 128, 0, c->st>>>(c->ncells, c->cell_start, c->cell_atoms, gate);
  c->launches += 4;
  if (c->mode == CM3D_NB_MIXED) {
    k_sorted_init<<<grid_for(n, B), B, 0, c->st>>>(n, c->cell_atoms, cimg, dhmat, c->nc[0], c->nc[1],
                                                    c->nc[2], c->itype, c->rank, c->styp, c->corner, gate);
    c->launches++;
  }
  ListParams P = params(c);
  k_list_count<<<grid_for(n, 128), 128, 0, c->st>>>(P, c->cell_atoms, c->cell_start, c->pos, c->itype, c->map,
                                                     c->icut, c->q, c->excl_off, c->excl_idx, c->cexcl_off,
                                                     c->cexcl_idx, cimg, c->ninter, c->cnt, gate);
  k_scan<int, long long><<<dim3(1, 5), 1024, 0, c->st>>>(c->cnt, c->off, c->ltot, n, gate);
  c->launches += 2;
  CKL(c);
  if (!device_flag) {
    CK(cudaMemcpyAsync(c->h_ltot, c->ltot, sizeof(long long) * LT_COUNT, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int k = 0; k < LT_COUNT; k++) {
      int rc = grow(c, k, c->h_ltot[k] > 0 ? c->h_ltot[k] : 1);
      if (rc) return rc;
      c->hcount[k] = c->h_ltot[k];
    }
    P = params(c);
  }
  k_list_fill<<<grid_for(n, 128), 128, 0, c->st>>>(P, c->cell_atoms, c->cell_start, c->pos, c->itype, c->map,
                                                    c->icut, c->q, c->excl_off, c->excl_idx, c->cexcl_off,
                                                    c->cexcl_idx, cimg, c->ninter, c->off, c->ltot, c->rank,
                                                    c->lst[0], c->lst[1], c->lst[2], c->lst[3], c->nbr,
                                                    c->stat, device_flag ? c->istate + IS_HALT : nullptr, gate);
  k_snapshot<<<grid_for(3LL * n, B), B, 0, c->st>>>(3 * n, c->pos, c->dxn, gate, c->istate, c->stat);
  c->launches += 2;
  CKL(c);
  tend(c, 2, e0);
  if (!device_flag) {
    c->lists_built = true;
    c->rebuilds_host++;
  }
  return CM3D_NB_OK;
}

}  // namespace cm3d
