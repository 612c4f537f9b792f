// Operator builder, device side: the upper-triangle CSR of an operator on a supercell,
// written row by row from the plan of tbmodel.cu (the reference builds it by inserting
// every replicated hopping into a std::multimap keyed by strings and handing the list to
// Eigen, utilities/wannier2sparse/src/hopping_list.cpp:158-285).
//
// Three passes over the rows, none of which stores per-row counts:
//   k_row_totals  rows' upper-triangle entry counts summed per block of 4096 rows
//   k_scan_totals exclusive scan of the block sums (one CTA); the total is the nnz
//   k_rowptr      counts again, block-local scan, rowptr written
// then k_fill writes every (cell, key) entry that lies in the upper triangle straight to
// its place: its rank in the row's column order comes from the rotation tree of the plan,
// so no sort and no atomics are needed and the output is deterministic.  The fill is a
// streaming write of 20 bytes per entry (column + complex value): HBM-bound.
#include <algorithm>
#include <cstring>
#include <memory>

#include "w2s_rows.cuh"

namespace linqt {
namespace w2s {

// plan tables in one device allocation
struct DevPlan {
  int device = -1;
  void *blob = nullptr;
  PlanView v{};
  void release() {
    if (blob) {
      cudaSetDevice(device);
      cudaFree(blob);
    }
    blob = nullptr;
  }
  ~DevPlan() { release(); }
};

namespace {

constexpr int kScanThreads = 256;
constexpr int kFillThreads = 256;
// shared memory per CTA of the fill, below the default dynamic limit; a sweep of 16-48 KB
// and of 2-8 cells per CTA (18-orbital model, 128 x 128 cells) moved the build by < 5 %
constexpr long kFillSmem = 48 * 1024;

// inclusive scan across the block (kScanThreads threads); returns the block total in *tot
__device__ long long block_inclusive_scan(long long x, long long *tot) {
  __shared__ long long warp_tot[kScanThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    long long w = lane < kScanThreads / 32 ? warp_tot[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kScanThreads / 32) warp_tot[lane] = w;
  }
  __syncthreads();
  const long long before = wid ? warp_tot[wid - 1] : 0;
  *tot = warp_tot[kScanThreads / 32 - 1];
  __syncthreads();
  return x + before;
}

// ITEMS consecutive rows per thread, ITEMS * kScanThreads per block
template <int ITEMS>
__global__ void __launch_bounds__(kScanThreads) k_row_totals(PlanView p, long long *bsum) {
  const long base = (long)blockIdx.x * kScanThreads * ITEMS + (long)threadIdx.x * ITEMS;
  long long s = 0;
#pragma unroll 4
  for (int i = 0; i < ITEMS; ++i)
    if (base + i < p.n) s += row_count(p, base + i);
  long long tot;
  block_inclusive_scan(s, &tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

// exclusive scan of nb block sums in place; bsum[nb] = total
__global__ void __launch_bounds__(kScanThreads) k_scan_totals(long long *bsum, int nb) {
  long long carry = 0;
  for (int b0 = 0; b0 < nb; b0 += kScanThreads) {
    const int i = b0 + threadIdx.x;
    const long long v = i < nb ? bsum[i] : 0;
    long long tot;
    const long long inc = block_inclusive_scan(v, &tot);
    if (i < nb) bsum[i] = carry + inc - v;
    carry += tot;
  }
  if (threadIdx.x == 0) bsum[nb] = carry;
}

template <int ITEMS>
__global__ void __launch_bounds__(kScanThreads) k_rowptr(PlanView p, const long long *boff, int *rowptr) {
  const long base = (long)blockIdx.x * kScanThreads * ITEMS + (long)threadIdx.x * ITEMS;
  int c[ITEMS];
  long long s = 0;
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    c[i] = base + i < p.n ? row_count(p, base + i) : 0;
    s += c[i];
  }
  long long tot;
  long long run = boff[blockIdx.x] + block_inclusive_scan(s, &tot) - s;
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    if (base + i < p.n) rowptr[base + i] = (int)run;
    run += c[i];
  }
  if (base <= p.n - 1 && p.n - 1 < base + ITEMS) rowptr[p.n] = (int)boff[gridDim.x];
}

// one thread per (cell, key): items i = s * K + t
template <class Idx>
__global__ void __launch_bounds__(256) k_fill(PlanView p, const int *__restrict__ rowptr, int *__restrict__ col,
                                              double2 *__restrict__ val) {
  const Idx total = (Idx)p.ncells * (Idx)p.K;
  const Idx stride = (Idx)gridDim.x * blockDim.x;
  for (Idx i = (Idx)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    const Idx s = i / (Idx)p.K;
    const int t = (int)(i - s * (Idx)p.K);
    long pos, c;
    if (!item_entry(p, rowptr, (long)s, t, pos, c)) continue;  // lower triangle: not stored
    col[pos] = (int)c;
    val[pos] = __ldg(&p.kval[t]);
  }
}

// one CTA per group of cpb cells: the cells' tables go to shared memory (their coordinates
// first), then every key of every cell is placed.  With at least as many keys per cell as
// threads, a thread loads a key once and places it in all cpb cells; otherwise the
// (cell, key) items are walked with a fixed stride (no division per item).
__global__ void __launch_bounds__(kFillThreads) k_fill_cells(PlanView p, const int *__restrict__ rowptr,
                                                             int *__restrict__ col, double2 *__restrict__ val,
                                                             int cpb) {
  extern __shared__ int tabs[];
  int *xyz = tabs;               // 3 per cell
  int *tab0 = tabs + 3 * cpb;    // cell tables
  const int per_cell = cell_table_size(p), NN = cell_table_items(p), K = p.K;
  const int qn = blockDim.x / NN, rn = blockDim.x % NN;
  const int c0n = threadIdx.x / NN, j0 = threadIdx.x % NN;
  for (long base = (long)blockIdx.x * cpb; base < p.ncells; base += (long)gridDim.x * cpb) {
    const int ncell = (int)min((long)cpb, p.ncells - base);
    for (int c = threadIdx.x; c < ncell; c += blockDim.x)
      cell_coords(p, base + c, xyz[3 * c], xyz[3 * c + 1], xyz[3 * c + 2]);
    __syncthreads();
    for (int c = c0n, j = j0; c < ncell;) {
      cell_table_entry(p, base + c, xyz[3 * c], xyz[3 * c + 1], xyz[3 * c + 2], j, rowptr, tab0 + c * per_cell);
      c += qn;
      j += rn;
      if (j >= NN) {
        j -= NN;
        c++;
      }
    }
    __syncthreads();
    if (K >= (int)blockDim.x) {
      // the next key's data is requested before this key is placed
      int t = threadIdx.x;
      int4 k = __ldg(&p.kpack[t]);
      int go = __ldg(&p.kgo[t]);
      double2 v = __ldg(&p.kval[t]);
      for (; t < K; t += blockDim.x) {
        const int tn = t + blockDim.x < K ? t + blockDim.x : t;
        const int4 kn = __ldg(&p.kpack[tn]);
        const int gon = __ldg(&p.kgo[tn]);
        const double2 vn = __ldg(&p.kval[tn]);
        for (int c = 0; c < ncell; ++c) {
          long pos, cc;
          if (key_place(p, k, go, tab0 + c * per_cell, pos, cc)) {
            col[pos] = (int)cc;
            val[pos] = v;
          }
        }
        k = kn;
        go = gon;
        v = vn;
      }
    } else {
      const int qk = blockDim.x / K, rk = blockDim.x % K;
      for (int c = threadIdx.x / K, t = threadIdx.x % K; c < ncell;) {
        long pos, cc;
        if (key_entry(p, t, tab0 + c * per_cell, pos, cc)) {
          col[pos] = (int)cc;
          val[pos] = __ldg(&p.kval[t]);
        }
        c += qk;
        t += rk;
        if (t >= K) {
          t -= K;
          c++;
        }
      }
    }
    __syncthreads();
  }
}

template <class T>
size_t put(std::vector<char> &blob, const std::vector<T> &v) {
  const size_t off = (blob.size() + 255) & ~(size_t)255;
  blob.resize(off + std::max<size_t>(1, v.size()) * sizeof(T), 0);
  if (!v.empty()) std::memcpy(blob.data() + off, v.data(), v.size() * sizeof(T));
  return off;
}

void upload(const Plan &pl, int device, DevPlan &d) {
  std::vector<char> blob;
  const size_t o_gk = put(blob, pl.grp_key0), o_gz = put(blob, pl.grp_z0), o_kz = put(blob, pl.kz),
               o_ky = put(blob, pl.ky), o_kx = put(blob, pl.kx), o_kl = put(blob, pl.kleaf), o_ko = put(blob, pl.ko1),
               o_kg = put(blob, pl.kgrp), o_zn = put(blob, pl.zn), o_yn = put(blob, pl.yn), o_xn = put(blob, pl.xn),
               o_kv = put(blob, pl.kval), o_kp = put(blob, pl.kpack), o_kgo = put(blob, pl.kgo);
  d.release();
  d.device = device;
  LQ_CUDA(cudaSetDevice(device));
  LQ_CUDA(cudaMalloc(&d.blob, blob.size()));
  LQ_CUDA(cudaMemcpy(d.blob, blob.data(), blob.size(), cudaMemcpyHostToDevice));
  char *b = (char *)d.blob;
  PlanView &v = d.v;
  v.wbb = pl.wbb;
  v.dx = pl.dims[0];
  v.dy = pl.dims[1];
  v.dz = pl.dims[2];
  v.K = pl.keys();
  v.ncells = pl.ncells;
  v.n = pl.n;
  v.grp_key0 = (const int *)(b + o_gk);
  v.grp_z0 = (const int *)(b + o_gz);
  v.kz = (const int *)(b + o_kz);
  v.ky = (const int *)(b + o_ky);
  v.kx = (const int *)(b + o_kx);
  v.kleaf = (const int *)(b + o_kl);
  v.ko1 = (const int *)(b + o_ko);
  v.kgrp = (const int *)(b + o_kg);
  v.zn = (const Node *)(b + o_zn);
  v.yn = (const Node *)(b + o_yn);
  v.xn = (const Node *)(b + o_xn);
  v.kval = (const double2 *)(b + o_kv);
  v.kpack = (const int4 *)(b + o_kp);
  v.kgo = (const int *)(b + o_kgo);
  v.nz = (int)pl.zn.size();
  v.ny = (int)pl.yn.size();
  v.nx = (int)pl.xn.size();
}

}  // namespace

// rowptr pass: returns nnz (rowptr left in rowptr_dev when it is not null)
template <int ITEMS>
static long count_rows_t(Session *s, const PlanView &v, int *rowptr_dev) {
  const long rows_per_block = (long)kScanThreads * ITEMS;
  const long nb = (v.n + rows_per_block - 1) / rows_per_block;
  LQ_REQUIRE(nb < 0x7fffffffL, "supercell too large");
  long long *bsum = (long long *)s->get("w2s_block_sums", sizeof(long long) * (nb + 1));
  PhaseScope ph(s, PH_OTHER);
  k_row_totals<ITEMS><<<(unsigned)nb, kScanThreads, 0, s->stream>>>(v, bsum);
  LQ_LAUNCHED();
  k_scan_totals<<<1, kScanThreads, 0, s->stream>>>(bsum, (int)nb);
  LQ_LAUNCHED();
  long long total = 0;
  LQ_CUDA(cudaMemcpyAsync(&total, bsum + nb, sizeof total, cudaMemcpyDeviceToHost, s->stream));
  LQ_CUDA(cudaStreamSynchronize(s->stream));
  LQ_REQUIRE(total <= 0x7fffffffLL, "the supercell operator has more than 2^31-1 stored entries");
  if (rowptr_dev) {
    k_rowptr<ITEMS><<<(unsigned)nb, kScanThreads, 0, s->stream>>>(v, bsum, rowptr_dev);
    LQ_LAUNCHED();
    ph.launches(3);
  } else {
    ph.launches(2);
  }
  return (long)total;
}

// rowptr pass: returns nnz (rowptr left in rowptr_dev when it is not null).  16 rows per
// thread, or 2 when that would leave SMs idle.
static long count_rows(Session *s, const PlanView &v, int *rowptr_dev) {
  if (v.n >= (long)kScanThreads * 16 * 2 * s->sm_count) return count_rows_t<16>(s, v, rowptr_dev);
  return count_rows_t<2>(s, v, rowptr_dev);
}

static void fill_rows(Session *s, const PlanView &v, const int *rowptr_dev, int *col_dev, double2 *val_dev) {
  if (v.K == 0 || v.ncells == 0) return;
  PhaseScope ph(s, PH_OTHER);
  const long table = 4L * (cell_table_size(v) + 3);
  if (table <= kFillSmem) {
    // cells per CTA: enough keys to keep the threads busy (4 cells when a thread places one
    // key in every cell), within the shared-memory budget
    const long by_smem = kFillSmem / table;
    const long want = v.K >= kFillThreads ? 4L : std::max(1L, (16L * kFillThreads + v.K - 1) / v.K);
    const int cpb = (int)std::max(1L, std::min(std::min(by_smem, want), v.ncells));
    const long blocks = (v.ncells + cpb - 1) / cpb;
    const unsigned grid = (unsigned)std::min<long>(blocks, (long)s->sm_count * 8);
    k_fill_cells<<<grid, kFillThreads, (size_t)(table * cpb), s->stream>>>(v, rowptr_dev, col_dev, val_dev, cpb);
  } else {
    const long total = v.ncells * (long)v.K;
    const long want = (total + 255) / 256;
    const unsigned grid = (unsigned)std::min<long>(want, (long)s->sm_count * 16);
    if (total < 0x7fffffffL)
      k_fill<unsigned><<<grid, 256, 0, s->stream>>>(v, rowptr_dev, col_dev, val_dev);
    else
      k_fill<unsigned long long><<<grid, 256, 0, s->stream>>>(v, rowptr_dev, col_dev, val_dev);
  }
  LQ_LAUNCHED();
  ph.launches(1);
}

}  // namespace w2s
}  // namespace linqt

using namespace linqt;

struct linqt_tbmodel {
  w2s::Model m;
  std::mutex mu;
  // the last plan built for a named operator (NAME.OP files are read afresh every call)
  std::string key;
  w2s::Plan plan;
  w2s::DevPlan dev;
};

namespace {

const w2s::PlanView &plan_for(linqt_tbmodel *m, Session *s, const char *op, const int dims[3]) {
  LQ_REQUIRE(op && dims, "NULL argument");
  std::string o(op);
  const bool builtin = w2s::is_builtin_op(o);
  std::string key = o + "|" + std::to_string(dims[0]) + "x" + std::to_string(dims[1]) + "x" +
                    std::to_string(dims[2]) + "@" + std::to_string(s->device);
  if (builtin && key == m->key && m->dev.blob) return m->dev.v;
  m->plan = w2s::make_plan(w2s::operator_list(m->m, o), m->m.num_wann, dims);
  w2s::upload(m->plan, s->device, m->dev);
  m->key = builtin ? key : std::string();
  return m->dev.v;
}

// the upper CSR in session workspaces; returns nnz
long build_on_device(linqt_tbmodel *m, Session *s, const char *op, const int dims[3], int **rp, int **cl,
                     double2 **vl) {
  const w2s::PlanView &v = plan_for(m, s, op, dims);
  *rp = (int *)s->get("w2s_rowptr", sizeof(int) * (v.n + 1));
  const long nnz = w2s::count_rows(s, v, *rp);
  *cl = (int *)s->get("w2s_col", sizeof(int) * std::max(1L, nnz));
  *vl = (double2 *)s->get("w2s_val", sizeof(double2) * std::max(1L, nnz));
  w2s::fill_rows(s, v, *rp, *cl, *vl);
  return nnz;
}

void to_host(linqt_tbmodel *m, Session *s, const char *op, const int dims[3], long &n, std::vector<int> &rowptr,
             std::vector<int> &col, std::vector<double2> &val) {
  int *rp, *cl;
  double2 *vl;
  const long nnz = build_on_device(m, s, op, dims, &rp, &cl, &vl);
  n = m->dev.v.n;
  rowptr.resize(n + 1);
  col.resize(nnz);
  val.resize(nnz);
  LQ_CUDA(cudaMemcpyAsync(rowptr.data(), rp, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s->stream));
  if (nnz) {
    LQ_CUDA(cudaMemcpyAsync(col.data(), cl, sizeof(int) * nnz, cudaMemcpyDeviceToHost, s->stream));
    LQ_CUDA(cudaMemcpyAsync(val.data(), vl, sizeof(double2) * nnz, cudaMemcpyDeviceToHost, s->stream));
  }
  LQ_CUDA(cudaStreamSynchronize(s->stream));
}

}  // namespace

extern "C" {

int linqt_tbmodel_load(const char *label, linqt_tbmodel **out) {
  return guarded([&] {
    LQ_REQUIRE(label && out, "NULL argument");
    std::unique_ptr<linqt_tbmodel> h(new linqt_tbmodel);
    h->m = w2s::load_model(label);
    *out = h.release();
  });
}

int linqt_tbmodel_destroy(linqt_tbmodel *m) {
  return guarded([&] { delete m; });
}

int linqt_tbmodel_info(const linqt_tbmodel *m, int *num_orbitals, long *num_hoppings) {
  return guarded([&] {
    LQ_REQUIRE(m, "NULL model");
    if (num_orbitals) *num_orbitals = m->m.num_wann;
    if (num_hoppings) *num_hoppings = (long)m->m.hops.size();
  });
}

int linqt_supercell_csr(linqt_session *s, linqt_tbmodel *m, const char *op, const int cell_dim[3], int *n, long *nnz,
                        int *rowptr, int *col, double *val, long capacity) {
  return guarded([&] {
    LQ_REQUIRE(m && n && nnz, "NULL argument");
    Session *r = resolve(s);
    std::lock_guard<std::mutex> g(m->mu);
    if (!rowptr) {  // size query
      const w2s::PlanView &v = plan_for(m, r, op, cell_dim);
      *n = (int)v.n;
      *nnz = w2s::count_rows(r, v, nullptr);
      return;
    }
    int *rp, *cl;
    double2 *vl;
    const long k = build_on_device(m, r, op, cell_dim, &rp, &cl, &vl);
    const long N = m->dev.v.n;
    *n = (int)N;
    *nnz = k;
    LQ_REQUIRE(capacity >= k, "capacity " + std::to_string(capacity) + " is below the " + std::to_string(k) +
                                  " stored entries");
    LQ_REQUIRE(k == 0 || (col && val), "NULL col/val");
    LQ_CUDA(cudaMemcpyAsync(rowptr, rp, sizeof(int) * (N + 1), cudaMemcpyDeviceToHost, r->stream));
    if (k) {
      LQ_CUDA(cudaMemcpyAsync(col, cl, sizeof(int) * k, cudaMemcpyDeviceToHost, r->stream));
      LQ_CUDA(cudaMemcpyAsync(val, vl, sizeof(double2) * k, cudaMemcpyDeviceToHost, r->stream));
    }
    LQ_CUDA(cudaStreamSynchronize(r->stream));
  });
}

int linqt_supercell_csr_dev(linqt_session *s, linqt_tbmodel *m, const char *op, const int cell_dim[3], int *n,
                            long *nnz, int *rowptr_dev, int *col_dev, double *val_dev, long capacity) {
  return guarded([&] {
    LQ_REQUIRE(m && n && nnz && rowptr_dev, "NULL argument");
    Session *r = resolve(s);
    std::lock_guard<std::mutex> g(m->mu);
    const w2s::PlanView &v = plan_for(m, r, op, cell_dim);
    *n = (int)v.n;
    const long k = w2s::count_rows(r, v, rowptr_dev);
    *nnz = k;
    LQ_REQUIRE(capacity >= k, "capacity " + std::to_string(capacity) + " is below the " + std::to_string(k) +
                                  " stored entries");
    LQ_REQUIRE(k == 0 || (col_dev && val_dev), "NULL col/val");
    w2s::fill_rows(r, v, rowptr_dev, col_dev, (double2 *)val_dev);
  });
}

int linqt_supercell_write_csr(linqt_session *s, linqt_tbmodel *m, const char *op, const int cell_dim[3],
                              const char *path) {
  return guarded([&] {
    LQ_REQUIRE(m && path, "NULL argument");
    Session *r = resolve(s);
    std::lock_guard<std::mutex> g(m->mu);
    long N;
    std::vector<int> rp, cl;
    std::vector<double2> vl;
    to_host(m, r, op, cell_dim, N, rp, cl, vl);
    w2s::write_csr_text(path, N, rp, cl, vl);
  });
}

int linqt_supercell_operator(linqt_session *s, linqt_tbmodel *m, const char *op, const int cell_dim[3],
                             linqt_op **out) {
  return guarded([&] {
    LQ_REQUIRE(m && out, "NULL argument");
    Session *r = resolve(s);
    std::lock_guard<std::mutex> g(m->mu);
    std::unique_ptr<linqt_op> h(new linqt_op);
    DeviceOp &d = h->op;
    long N;
    to_host(m, r, op, cell_dim, N, d.up_rowptr, d.up_col, d.up_val);
    d.device = r->device;
    d.n = (int)N;
    d.hermitian = true;  // the file's semantics: upper triangle, the solver mirrors it
    d.upload();
    *out = h.release();
  });
}

}  // extern "C"
