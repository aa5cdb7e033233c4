// Solver runtime: device-side set-up of the operator and the multigrid hierarchy, V-cycle, CG with
// device-resident scalars (graph-captured iterations), FP64 iterative refinement, and the C ABI.
//
// Reference algorithm: fe/gmg.py (GMG + PCG), rb/gpusolve.py (GPU variant: FP64 CG, FP32 V-cycle,
// dense FP64 coarse solve, rigid-mode correction), rb/splitfe.py:123-158 (split-node solve).
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <future>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "coarse.cuh"
#include "dense.cuh"
#include "fine.cuh"
#include "rigid.cuh"
#include "vec.cuh"

namespace feb {

static thread_local char g_err[512] = "";
static std::atomic<long long> g_launches{0};

// Set-up profiling (FEB_PROFILE_SETUP=1): wall time of each set-up segment, device work included (the
// stream is synchronised at every mark), printed to stderr when feb_create returns.
struct SetupProfile {
  bool on = false;
  std::vector<std::pair<std::string, double>> marks;
  std::chrono::steady_clock::time_point t0;
  void start(bool enable) {
    on = enable;
    marks.clear();
    t0 = std::chrono::steady_clock::now();
  }
  void mark(const char* what, cudaStream_t s) {
    if (!on) return;
    cudaStreamSynchronize(s);
    auto t = std::chrono::steady_clock::now();
    marks.emplace_back(what, std::chrono::duration<double, std::milli>(t - t0).count());
    t0 = t;
  }
  void print() const {
    if (!on) return;
    for (const auto& m : marks) std::fprintf(stderr, "feb setup %-28s %8.3f ms\n", m.first.c_str(), m.second);
  }
};
thread_local SetupProfile g_prof;

// kernels recorded into a graph by this thread are not launches: they count when the graph runs
thread_local bool g_capturing = false;
void note_launch(int n) {
  if (!g_capturing) g_launches.fetch_add(n, std::memory_order_relaxed);
}

int set_dyn_smem(const void* kernel, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> done;   // (kernel, device) -> bytes set
  int dev = 0;
  FEB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  auto it = done.find({kernel, dev});
  if (it != done.end() && it->second >= bytes) return FEB_OK;
  FEB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done[{kernel, dev}] = bytes;
  return FEB_OK;
}

void set_last_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

namespace {

constexpr int kMaxLevels = 8;
constexpr int kTermDotBufs = 2 * 9 - 1;   // V-cycle term-dot buffers of a level for Chebyshev degrees <= 9

// ------------------------------------------------------------------------------------------------ memory
// Set-up uploads go through one process-wide pinned staging ring: a host copy into pinned memory, then an
// asynchronous DMA, so an upload neither stalls the host on the stream nor runs at pageable-copy speed.  Each
// staged copy records an event; before the ring wraps, the host waits for the copies issued since the last
// wrap (any stream).  Requests larger than the ring are copied directly.
class PinnedStaging {
 public:
  int copy(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    std::lock_guard<std::mutex> lock(mu_);
    if (!buf_) {
      if (cudaMallocHost(&buf_, kCap) != cudaSuccess) { buf_ = nullptr; cudaGetLastError(); }
    }
    if (!buf_ || bytes > kCap) {
      FEB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
      return FEB_OK;
    }
    if (off_ + bytes > kCap) {      // wrap: every copy out of the ring so far has to be done
      for (size_t i = 0; i < used_; ++i) FEB_CUDA(cudaEventSynchronize(ev_[i]));
      used_ = 0;
      off_ = 0;
    }
    if (used_ == ev_.size()) {
      cudaEvent_t e;
      FEB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      ev_.push_back(e);
    }
    char* at = static_cast<char*>(buf_) + off_;
    std::memcpy(at, src, bytes);
    FEB_CUDA(cudaMemcpyAsync(dst, at, bytes, cudaMemcpyHostToDevice, s));
    FEB_CUDA(cudaEventRecord(ev_[used_++], s));
    off_ += (bytes + 255) & ~size_t(255);
    return FEB_OK;
  }

 private:
  static constexpr size_t kCap = size_t(32) << 20;
  std::mutex mu_;
  void* buf_ = nullptr;             // kept until the process exits
  size_t off_ = 0, used_ = 0;
  std::vector<cudaEvent_t> ev_;
};
PinnedStaging g_staging;

class Pool {
 public:
  explicit Pool(cudaStream_t s) : s_(s) {}
  ~Pool() { release(); }
  template <typename T>
  int alloc(T** p, size_t n) {
    *p = nullptr;
    if (n == 0) return FEB_OK;
    cudaError_t e = cudaMallocAsync((void**)p, n * sizeof(T), s_);
    if (e != cudaSuccess) {
      set_last_error("cudaMallocAsync(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? FEB_ERR_NOMEM : FEB_ERR_CUDA;
    }
    ptrs_.push_back((void*)*p);
    return FEB_OK;
  }
  template <typename T>
  int zeros(T** p, size_t n) {
    FEB_TRY(alloc(p, n));
    if (n) FEB_CUDA(cudaMemsetAsync(*p, 0, n * sizeof(T), s_));
    return FEB_OK;
  }
  template <typename T>
  int upload(T** p, const T* h, size_t n) {
    FEB_TRY(alloc(p, n));
    if (n) FEB_TRY(g_staging.copy(*p, h, n * sizeof(T), s_));
    return FEB_OK;
  }
  void free(void* p) {
    if (!p) return;
    auto it = std::find(ptrs_.begin(), ptrs_.end(), p);
    if (it != ptrs_.end()) {
      cudaFreeAsync(p, s_);
      ptrs_.erase(it);
    }
  }
  void release() {
    for (void* p : ptrs_) cudaFreeAsync(p, s_);
    ptrs_.clear();
  }

 private:
  cudaStream_t s_;
  std::vector<void*> ptrs_;
};

// ------------------------------------------------------------------------------------------------ host helpers
struct AxisHost {
  int nf = 0, nc = 0;
  std::vector<int> ca, cb, cidx, iv_first, iv_count;
  std::vector<double> wa, wb, coarse;
};

// 1-D prolongation from every other node plus the last one with linear weights (fe/gmg.py:7-26)
int env_flag(const char* name);   // 1 when the variable is set to anything but "" or "0"

AxisHost make_axis(const std::vector<double>& c) {
  AxisHost A;
  const int n = (int)c.size();
  A.nf = n;
  for (int i = 0; i < n; i += 2) A.cidx.push_back(i);
  if (A.cidx.back() != n - 1) A.cidx.push_back(n - 1);
  A.nc = (int)A.cidx.size();
  A.ca.resize(n); A.cb.resize(n); A.wa.resize(n); A.wb.resize(n);
  std::vector<int> pos(n, -1);
  for (int J = 0; J < A.nc; ++J) pos[A.cidx[J]] = J;
  for (int i = 0; i < n; ++i) {
    if (pos[i] >= 0) {
      A.ca[i] = A.cb[i] = pos[i]; A.wa[i] = 1.0; A.wb[i] = 0.0;
    } else {
      int a = (i - 1) / 2, b = a + 1;
      double w = (c[i] - c[A.cidx[a]]) / (c[A.cidx[b]] - c[A.cidx[a]]);
      A.ca[i] = a; A.cb[i] = b; A.wa[i] = 1.0 - w; A.wb[i] = w;
    }
  }
  for (int J = 0; J + 1 < A.nc; ++J) {
    A.iv_first.push_back(A.cidx[J]);
    A.iv_count.push_back(A.cidx[J + 1] - A.cidx[J]);
  }
  for (int J = 0; J < A.nc; ++J) A.coarse.push_back(c[A.cidx[J]]);
  return A;
}

// host sparse entries on dofs (3 node + comp) of one level
struct Entries {
  std::vector<int64_t> r, c;
  std::vector<double> v;
  size_t size() const { return v.size(); }
};

// Stable LSD radix sort of key[0, n) (idx carried along), 11-bit digits (the histogram stays in L1), digits
// constant over all keys skipped; k2 / i2 are scratch of the same length.  The result ends in key / idx.
void radix_range(uint64_t* key, uint32_t* idx, uint64_t* k2, uint32_t* i2, size_t n) {
  uint64_t any_or = 0, any_and = ~0ull;
  for (size_t i = 0; i < n; ++i) { any_or |= key[i]; any_and &= key[i]; }
  constexpr int kBits = 11;
  constexpr uint64_t kMask = (1u << kBits) - 1;
  uint32_t cnt[size_t(1) << kBits];
  uint64_t *ka = key, *kb = k2;
  uint32_t *ia = idx, *ib = i2;
  for (int shift = 0; shift < 64; shift += kBits) {
    if ((((any_or ^ any_and) >> shift) & kMask) == 0) continue;
    std::fill(cnt, cnt + (size_t(1) << kBits), 0u);
    for (size_t i = 0; i < n; ++i) cnt[(ka[i] >> shift) & kMask]++;
    uint32_t sum = 0;
    for (auto& c : cnt) { const uint32_t t = c; c = sum; sum += t; }
    for (size_t i = 0; i < n; ++i) {
      const uint32_t at = cnt[(ka[i] >> shift) & kMask]++;
      kb[at] = ka[i];
      ib[at] = ia[i];
    }
    std::swap(ka, kb);
    std::swap(ia, ib);
  }
  if (ka != key) {
    std::copy(ka, ka + n, key);
    std::copy(ia, ia + n, idx);
  }
}

// Sorts entries by (row, col) and sums duplicates (in input order): the packed key row << 32 | col (dofs < 2^31,
// feb_create checks 3 nnode_total) radix-sorted.  Large inputs are first cut into 4 key ranges (splitters from
// the quartiles of a sample; a stable counting pass), sorted on 4 threads; the result is the same as one sort.
void coo_merge(Entries& E) {
  const size_t n = E.size();
  if (n == 0) return;
  std::vector<uint64_t> key(n), k2(n);
  std::vector<uint32_t> idx(n), i2(n);
  for (size_t i = 0; i < n; ++i) {
    key[i] = ((uint64_t)E.r[i] << 32) | (uint32_t)E.c[i];
    idx[i] = (uint32_t)i;
  }
  constexpr int kParts = 4;
  if (n >= 32768 && std::thread::hardware_concurrency() >= (unsigned)kParts) {
    // key ranges of about equal size from the quartiles of a sample (equal keys share a range)
    std::vector<uint64_t> smp;
    const size_t step = std::max<size_t>(1, n / 4096);
    for (size_t i = 0; i < n; i += step) smp.push_back(key[i]);
    std::sort(smp.begin(), smp.end());
    uint64_t split[kParts - 1];
    for (int p = 1; p < kParts; ++p) split[p - 1] = smp[smp.size() * p / kParts];
    auto part = [&](size_t i) { return (int)(std::upper_bound(split, split + kParts - 1, key[i]) - split); };
    size_t off[kParts + 1] = {};
    for (size_t i = 0; i < n; ++i) off[part(i) + 1]++;
    for (int p = 0; p < kParts; ++p) off[p + 1] += off[p];
    size_t fill[kParts];
    std::copy(off, off + kParts, fill);
    for (size_t i = 0; i < n; ++i) {     // stable scatter into the row ranges
      const size_t at = fill[part(i)]++;
      k2[at] = key[i];
      i2[at] = idx[i];
    }
    key.swap(k2);
    idx.swap(i2);
    std::vector<std::thread> th;
    for (int p = 1; p < kParts; ++p)
      th.emplace_back(radix_range, key.data() + off[p], idx.data() + off[p], k2.data() + off[p], i2.data() + off[p],
                      off[p + 1] - off[p]);
    radix_range(key.data(), idx.data(), k2.data(), i2.data(), off[1]);
    for (auto& t : th) t.join();
  } else {
    radix_range(key.data(), idx.data(), k2.data(), i2.data(), n);
  }
  // rows and columns come back out of the sorted keys; only the values are gathered
  std::vector<double> vals(n);
  size_t m = 0;
  for (size_t t = 0; t < n; ++t) {
    const double v = E.v[idx[t]];
    if (t > 0 && key[t] == key[t - 1]) vals[m - 1] += v;
    else { k2[m] = key[t]; vals[m++] = v; }
  }
  E.r.resize(m); E.c.resize(m);
  for (size_t t = 0; t < m; ++t) { E.r[t] = (int64_t)(k2[t] >> 32); E.c[t] = (int64_t)(uint32_t)k2[t]; }
  vals.resize(m);
  E.v.swap(vals);
}

// supports of a node position along each axis
inline int supp(const AxisHost& A, int i, int (&J)[2], double (&w)[2]) {
  int n = 0;
  if (A.wa[i] != 0.0) { J[n] = A.ca[i]; w[n] = A.wa[i]; ++n; }
  if (A.cb[i] != A.ca[i] && A.wb[i] != 0.0) { J[n] = A.cb[i]; w[n] = A.wb[i]; ++n; }
  return n;
}

// P^T E P for entries E of a level whose node `pos` maps to grid positions (fnx, fny)
Entries project(const Entries& E, const AxisHost (&ax)[3], const std::vector<int64_t>& pos_of_node_copy,
                int64_t fnnode, int fnx, int fny) {
  Entries out;
  const int64_t cnx = ax[0].nc, cny = ax[1].nc;
  auto position = [&](int64_t node) { return node < fnnode ? node : pos_of_node_copy[node - fnnode]; };
  for (size_t e = 0; e < E.size(); ++e) {
    int64_t pr = position(E.r[e] / 3), pc = position(E.c[e] / 3);
    int ir[3] = {int(pr % fnx), int((pr / fnx) % fny), int(pr / ((int64_t)fnx * fny))};
    int ic[3] = {int(pc % fnx), int((pc / fnx) % fny), int(pc / ((int64_t)fnx * fny))};
    int Jr[3][2], Jc[3][2], nr[3], nc[3];
    double wr[3][2], wc[3][2];
    for (int d = 0; d < 3; ++d) { nr[d] = supp(ax[d], ir[d], Jr[d], wr[d]); nc[d] = supp(ax[d], ic[d], Jc[d], wc[d]); }
    for (int a = 0; a < nr[0]; ++a) for (int b = 0; b < nr[1]; ++b) for (int c = 0; c < nr[2]; ++c) {
      int64_t J = Jr[0][a] + cnx * (Jr[1][b] + cny * Jr[2][c]);
      double wJ = wr[0][a] * wr[1][b] * wr[2][c];
      for (int a2 = 0; a2 < nc[0]; ++a2) for (int b2 = 0; b2 < nc[1]; ++b2) for (int c2 = 0; c2 < nc[2]; ++c2) {
        int64_t K = Jc[0][a2] + cnx * (Jc[1][b2] + cny * Jc[2][c2]);
        out.r.push_back(3 * J + E.r[e] % 3);
        out.c.push_back(3 * K + E.c[e] % 3);
        out.v.push_back(wJ * wc[0][a2] * wc[1][b2] * wc[2][c2] * E.v[e]);
      }
    }
  }
  coo_merge(out);
  return out;
}

// Rank-1 terms lam_t v_t v_t^T of the extra matrix.  Non-local spring couplings (a ligament between two
// bones, a penalty over a face) are low-rank by construction, rb/replica3.py:68-86 and
// fe/solver.py:224-232 add k w w^T; carried as terms, a level's couplings are projected to the next level
// as vectors (P^T v, at most 8x the entries) instead of as outer products (64x the entries).
struct Terms {
  std::vector<double> lam;
  std::vector<int64_t> ptr{0};   // entries of term t: ptr[t] .. ptr[t+1]
  std::vector<int64_t> dof;      // level dofs, 3 node + comp
  std::vector<double> val;
  size_t size() const { return lam.size(); }
};

// Symmetric m x m matrix (row-major, modified) -> terms by LDL^T with diagonal pivoting.  Succeeds when
// the remainder after at most max_rank pivots vanishes (|entries| <= 1e-12 of the largest), which holds for
// sums of a few positive semidefinite springs; returns false otherwise (the caller keeps the entries).
// dofs maps the m local indices to level dofs.
bool factor_terms(std::vector<double>& A, int m, const std::vector<int64_t>& dofs, int max_rank, Terms& out) {
  double scale = 0.0;
  for (double a : A) scale = std::max(scale, std::fabs(a));
  if (scale == 0.0) return true;
  const double tol = 1e-12 * scale;
  std::vector<char> done(m, 0);
  Terms T;
  for (int step = 0; step < m; ++step) {
    int p = -1;
    double best = tol;
    for (int i = 0; i < m; ++i)
      if (!done[i] && std::fabs(A[(size_t)i * m + i]) > best) { best = std::fabs(A[(size_t)i * m + i]); p = i; }
    if (p < 0) break;
    if ((int)T.size() == max_rank) return false;
    const double d = A[(size_t)p * m + p];
    std::vector<double> l(m);
    for (int i = 0; i < m; ++i) l[i] = A[(size_t)i * m + p] / d;
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) A[(size_t)i * m + j] -= d * l[i] * l[j];
    done[p] = 1;
    T.lam.push_back(d);
    for (int i = 0; i < m; ++i)
      if (l[i] != 0.0) { T.dof.push_back(dofs[i]); T.val.push_back(l[i]); }
    T.ptr.push_back((int64_t)T.dof.size());
  }
  for (double a : A)
    if (std::fabs(a) > tol) return false;
  for (size_t t = 0; t < T.size(); ++t) {
    out.lam.push_back(T.lam[t]);
    for (int64_t e = T.ptr[t]; e < T.ptr[t + 1]; ++e) { out.dof.push_back(T.dof[e]); out.val.push_back(T.val[e]); }
    out.ptr.push_back((int64_t)out.dof.size());
  }
  return true;
}

// P^T v of every term (same node positions and supports as project())
Terms project_terms(const Terms& T, const AxisHost (&ax)[3], const std::vector<int64_t>& pos_of_node_copy,
                    int64_t fnnode, int fnx, int fny) {
  Terms out;
  const int64_t cnx = ax[0].nc, cny = ax[1].nc;
  auto position = [&](int64_t node) { return node < fnnode ? node : pos_of_node_copy[node - fnnode]; };
  std::vector<std::pair<int64_t, double>> acc;
  for (size_t t = 0; t < T.size(); ++t) {
    acc.clear();
    for (int64_t e = T.ptr[t]; e < T.ptr[t + 1]; ++e) {
      const int64_t p = position(T.dof[e] / 3);
      const int comp = int(T.dof[e] % 3);
      const int ip[3] = {int(p % fnx), int((p / fnx) % fny), int(p / ((int64_t)fnx * fny))};
      int J[3][2], n[3];
      double w[3][2];
      for (int d = 0; d < 3; ++d) n[d] = supp(ax[d], ip[d], J[d], w[d]);
      for (int a = 0; a < n[0]; ++a) for (int b = 0; b < n[1]; ++b) for (int c = 0; c < n[2]; ++c)
        acc.emplace_back(3 * (J[0][a] + cnx * (J[1][b] + cny * J[2][c])) + comp, w[0][a] * w[1][b] * w[2][c] * T.val[e]);
    }
    std::sort(acc.begin(), acc.end(), [](const std::pair<int64_t, double>& x, const std::pair<int64_t, double>& y) {
      return x.first < y.first;
    });
    for (size_t i = 0; i < acc.size();) {
      size_t j = i;
      double v = 0.0;
      for (; j < acc.size() && acc[j].first == acc[i].first; ++j) v += acc[j].second;
      if (v != 0.0) { out.dof.push_back(acc[i].first); out.val.push_back(v); }
      i = j;
    }
    out.lam.push_back(T.lam[t]);
    out.ptr.push_back((int64_t)out.dof.size());
  }
  return out;
}

// Connected components (over dofs) of the non-local entries; each component of at most kTermDofs dofs
// whose entries (every entry with both dofs in it, local ones included) factor into at most kTermRank
// rank-1 terms is moved to `terms`.  Returns the flags of the entries that the terms now represent.
constexpr int kTermDofs = 1024;
constexpr int kTermRank = 48;
std::vector<char> factor_nonlocal(const Entries& ex, const std::vector<char>& is_local, Terms& terms) {
  std::vector<char> taken(ex.size(), 0);
  std::vector<int64_t> nd;                        // dofs of the non-local entries, sorted
  for (size_t e = 0; e < ex.size(); ++e)
    if (!is_local[e]) { nd.push_back(ex.r[e]); nd.push_back(ex.c[e]); }
  if (nd.empty()) return taken;
  std::sort(nd.begin(), nd.end());
  nd.erase(std::unique(nd.begin(), nd.end()), nd.end());
  auto index = [&](int64_t d) {
    auto it = std::lower_bound(nd.begin(), nd.end(), d);
    return (it != nd.end() && *it == d) ? int(it - nd.begin()) : -1;
  };
  std::vector<int> parent(nd.size());
  for (size_t i = 0; i < nd.size(); ++i) parent[i] = (int)i;
  auto find = [&](int x) {
    while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; }
    return x;
  };
  for (size_t e = 0; e < ex.size(); ++e) {
    if (is_local[e]) continue;
    const int a = find(index(ex.r[e])), b = find(index(ex.c[e]));
    if (a != b) parent[std::max(a, b)] = std::min(a, b);
  }
  // components in the order of their smallest dof; entries with both dofs in one component
  std::vector<int> comp(nd.size(), -1), root_comp(nd.size(), -1);
  std::vector<std::vector<int64_t>> dofs;
  for (size_t i = 0; i < nd.size(); ++i) {
    const int r = find((int)i);
    if (root_comp[r] < 0) { root_comp[r] = (int)dofs.size(); dofs.emplace_back(); }
    comp[i] = root_comp[r];
    dofs[comp[i]].push_back(nd[i]);
  }
  std::vector<std::vector<size_t>> ents(dofs.size());
  for (size_t e = 0; e < ex.size(); ++e) {
    const int ia = index(ex.r[e]);
    if (ia < 0) continue;
    const int ib = index(ex.c[e]);
    if (ib >= 0 && comp[ia] == comp[ib]) ents[comp[ia]].push_back(e);
  }
  for (size_t cpt = 0; cpt < dofs.size(); ++cpt) {
    const std::vector<int64_t>& D = dofs[cpt];     // sorted (nd is sorted)
    const int m = (int)D.size();
    if (m > kTermDofs) continue;
    std::vector<double> A((size_t)m * m, 0.0);
    auto li = [&](int64_t d) { return int(std::lower_bound(D.begin(), D.end(), d) - D.begin()); };
    for (size_t e : ents[cpt]) A[(size_t)li(ex.r[e]) * m + li(ex.c[e])] += ex.v[e];
    if (factor_terms(A, m, D, kTermRank, terms))
      for (size_t e : ents[cpt]) taken[e] = 1;
  }
  return taken;
}

}  // namespace

// symmetric pseudo-inverse by cyclic Jacobi (numpy.linalg.pinv semantics: cutoff 1e-15 * max |eig|)
std::vector<double> sym_pinv(const std::vector<double>& A0, int n) {
  std::vector<double> A(A0), V(n * n, 0.0);
  for (int i = 0; i < n; ++i) V[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) { tot += A[i * n + j] * A[i * n + j]; if (i != j) off += A[i * n + j] * A[i * n + j]; }
    if (off <= 1e-30 * tot) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = A[p * n + q];
        if (std::fabs(apq) < 1e-300) continue;
        double theta = (A[q * n + q] - A[p * n + p]) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          double akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - s * akq;
          A[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          double apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - s * aqk;
          A[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double vkp = V[k * n + p], vkq = V[k * n + q];
          V[k * n + p] = c * vkp - s * vkq;
          V[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  double mx = 0.0;
  for (int i = 0; i < n; ++i) mx = std::max(mx, std::fabs(A[i * n + i]));
  std::vector<double> P(n * n, 0.0);
  for (int k = 0; k < n; ++k) {
    double ev = A[k * n + k];
    if (std::fabs(ev) <= 1e-15 * mx) continue;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) P[i * n + j] += V[i * n + k] * V[j * n + k] / ev;
  }
  return P;
}

namespace {

// ------------------------------------------------------------------------------------------------ cell set-up
template <int W>
__global__ void k_prepare_cells(int nx, int ny, int nz, const double* __restrict__ mat, int mode,
                                const uint8_t* __restrict__ active, const int64_t* __restrict__ cn,
                                double* __restrict__ mat_all, double* __restrict__ mat_s64, float* __restrict__ mat_s32,
                                uint8_t* __restrict__ irr_flag, uint8_t* __restrict__ used) {
  const int64_t ncell = (int64_t)nx * ny * nz;
  int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= ncell) return;
  int k = int(r % nz), j = int((r / nz) % ny), i = int(r / ((int64_t)nz * ny));
  int64_t xc = i + (int64_t)nx * (j + (int64_t)ny * k);
  const int64_t nx1 = nx + 1, ny1 = ny + 1;
  bool act = active[r] != 0;
  bool irr = false;
  if (act) {
    for (int l = 0; l < 8; ++l) {
      int64_t g = (i + (l & 1)) + nx1 * ((j + ((l >> 1) & 1)) + ny1 * (k + ((l >> 2) & 1)));
      int64_t node = cn ? cn[8 * r + l] : g;
      irr |= (node != g);
      used[node] = 1;
    }
  }
  double v[W];
  for (int q = 0; q < W; ++q) v[q] = (mode == MAT_ORTHO) ? mat[W * r + q] : mat[q * ncell + r];
  for (int q = 0; q < W; ++q) {
    double a = act ? v[q] : 0.0, s = (act && !irr) ? v[q] : 0.0;
    mat_all[W * xc + q] = a;
    mat_s64[W * xc + q] = s;
    mat_s32[W * xc + q] = float(s);
  }
  irr_flag[r] = (act && irr) ? 1 : 0;
}

template <int W>
__global__ void k_build_irregular(int nx, int ny, int nz, const int64_t* __restrict__ irr_ref, int nirr,
                                  const double* __restrict__ mat, int mode, const int64_t* __restrict__ cn,
                                  int* __restrict__ irr_cell, int* __restrict__ irr_nodes, double* __restrict__ m64,
                                  float* __restrict__ m32) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nirr) return;
  const int64_t ncell = (int64_t)nx * ny * nz;
  int64_t r = irr_ref[e];
  int k = int(r % nz), j = int((r / nz) % ny), i = int(r / ((int64_t)nz * ny));
  irr_cell[e] = int(i + (int64_t)nx * (j + (int64_t)ny * k));
  for (int l = 0; l < 8; ++l) irr_nodes[8 * e + l] = int(cn[8 * r + l]);
  for (int q = 0; q < W; ++q) {
    double v = (mode == MAT_ORTHO) ? mat[W * r + q] : mat[q * ncell + r];
    m64[W * e + q] = v;
    m32[W * e + q] = float(v);
  }
}

__global__ void k_orig_copy(const int64_t* __restrict__ orig, int64_t nnode, int64_t ntotal, int* __restrict__ out) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ntotal - nnode) return;
  out[e] = int(orig[nnode + e]);
}

// x += a y (y may alias x: x *= 1 + a; no restrict qualifiers for that reason)
__global__ void k_axpy_inplace(double* x, const double* y, int64_t n, double a) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) x[i] += a * y[i];
}

// Rigid groups, filtered on the device.  Group g's entries are cut into chunks of 1024 (one CTA per chunk and
// group): the count pass writes each chunk's number of used nodes and adds it to the group's count (a node id
// out of range sets *bad); the compaction pass writes the used nodes of the kept groups in their given order,
// each chunk at the group's destination offset plus the counts of the group's earlier chunks.
__global__ void __launch_bounds__(1024)
k_group_count(const int64_t* __restrict__ nodes, const int64_t* __restrict__ off, const uint8_t* __restrict__ used,
              int64_t ntotal, int ngroups, int nchunk, int* __restrict__ chunk_cnt, int* __restrict__ count,
              int* __restrict__ bad) {
  for (int g = blockIdx.y; g < ngroups; g += gridDim.y) {
    const int64_t e = off[g] + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int c = 0;
    if (e < off[g + 1]) {
      const int64_t n = nodes[e];
      if (n < 0 || n >= ntotal) atomicExch(bad, 1);
      else c = used[n] ? 1 : 0;
    }
    c = block_sum(c);
    if (threadIdx.x == 0) {
      chunk_cnt[(size_t)g * nchunk + blockIdx.x] = c;
      if (c) atomicAdd(count + g, c);
    }
    __syncthreads();   // block_sum's shared scratch is reused by the next group
  }
}

__global__ void __launch_bounds__(1024)
k_group_compact(const int64_t* __restrict__ nodes, const int64_t* __restrict__ off, const uint8_t* __restrict__ used,
                int ngroups, int nchunk, const int* __restrict__ chunk_cnt, const int* __restrict__ dst_off,
                int64_t* __restrict__ out) {
  __shared__ int warp_tot[32];
  __shared__ int prior_s;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int g = blockIdx.y; g < ngroups; g += gridDim.y) {
    if (dst_off[g] < 0) continue;       // dropped group (uniform over the CTA)
    const int64_t e0 = off[g] + (int64_t)blockIdx.x * blockDim.x;
    if (e0 >= off[g + 1]) continue;     // past the group's end (uniform)
    int prior = 0;                      // used nodes in the group's earlier chunks
    for (int q = threadIdx.x; q < (int)blockIdx.x; q += blockDim.x) prior += chunk_cnt[(size_t)g * nchunk + q];
    prior = block_sum(prior);
    if (threadIdx.x == 0) prior_s = prior;
    __syncthreads();
    prior = prior_s;
    const int64_t e = e0 + threadIdx.x;
    const bool keep = e < off[g + 1] && used[nodes[e]];
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    const int before = __popc(m & ((1u << lane) - 1u));
    if (lane == 0) warp_tot[w] = __popc(m);
    __syncthreads();
    int prefix = 0;
    for (int q = 0; q < w && q < nw; ++q) prefix += warp_tot[q];
    if (keep) out[dst_off[g] + prior + prefix + before] = nodes[e];
    __syncthreads();
  }
}

__global__ void k_masked_copy(const double* __restrict__ src, const uint8_t* __restrict__ used, int64_t n,
                              double* __restrict__ dst) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= 3 * n) return;
  dst[i] = used[i / 3] ? src[i] : 0.0;
}

__global__ void k_export(const double* __restrict__ x, const uint8_t* __restrict__ used, int64_t n,
                         double* __restrict__ U) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= 3 * n) return;
  U[i] = used[i / 3] ? x[i] : __longlong_as_double(0x7ff8000000000000LL);
}

struct Csr {
  int nrow = 0;
  int *row_dof = nullptr, *row_ptr = nullptr, *col = nullptr;
  double* v64 = nullptr;
  float* v32 = nullptr;
};

int upload_csr(Pool& pool, const Entries& E, Csr& C) {
  std::vector<int> rd, rp, cl;
  std::vector<double> v;
  std::vector<float> vf;
  cl.reserve(E.size()); v.reserve(E.size()); vf.reserve(E.size());
  for (size_t e = 0; e < E.size(); ++e) {
    if (rd.empty() || rd.back() != E.r[e]) { rd.push_back((int)E.r[e]); rp.push_back((int)e); }
    cl.push_back((int)E.c[e]);
    v.push_back(E.v[e]);
    vf.push_back((float)E.v[e]);
  }
  rp.push_back((int)E.size());
  C.nrow = (int)rd.size();
  if (C.nrow == 0) return FEB_OK;
  FEB_TRY(pool.upload(&C.row_dof, rd.data(), rd.size()));
  FEB_TRY(pool.upload(&C.row_ptr, rp.data(), rp.size()));
  FEB_TRY(pool.upload(&C.col, cl.data(), cl.size()));
  FEB_TRY(pool.upload(&C.v64, v.data(), v.size()));
  FEB_TRY(pool.upload(&C.v32, vf.data(), vf.size()));
  return FEB_OK;
}

struct Level {
  int nx = 0, ny = 0, nz = 0;             // node grid of this level
  int64_t nnode = 0, ntotal = 0;          // grid nodes, grid nodes + copies (level 0)
  int64_t ndof = 0;                       // 3 x used / kept nodes
  std::vector<double> coord[3];
  uint8_t* used = nullptr;
  double* A64 = nullptr;                  // full stencil [243][n] (levels >= 1, set-up only)
  double* S64 = nullptr;                  // symmetric half storage [126][n] (levels >= 1)
  float* S32 = nullptr;
  __half* S16 = nullptr;                  // 16-bit copy for the FP32 products (instead of S32), and its scale
  float* hscale = nullptr;                // [2]: the scale, then the largest |entry| (as bits) it was formed from
  int* node_ptr = nullptr;                // per-node CSR of the entries the stencil cannot hold
  int8_t* ent_r = nullptr;
  int* ent_col = nullptr;
  double* ent_v64 = nullptr;
  float* ent_v32 = nullptr;
  Entries nonlocal;                       // non-local entries kept as entries (projected entry by entry)
  Terms terms;                            // non-local couplings as rank-1 terms (projected as vectors)
  Entries sparse;                         // this level's entries outside the stencil (non-factored remainder)
  int nterms = 0;                         // device copy of `terms` and its per-node pairs (levels >= 1)
  int *t_ptr = nullptr, *t_dof = nullptr, *tn_ptr = nullptr, *tn_term = nullptr;
  double *t_val64 = nullptr, *t_lam64 = nullptr, *tn_coef64 = nullptr;
  float *t_val32 = nullptr, *t_lam32 = nullptr, *tn_coef32 = nullptr;
  double* Dinv64 = nullptr;
  float* Dinv32 = nullptr;
  double* tdot64 = nullptr;               // per-term dots of the current product (rank-1 terms)
  float* tdot32 = nullptr;
  // the V-cycle's term dots, formed by the kernels that write the level's vectors (TermAcc): buffer 0 the
  // iterate x, 1 .. deg-1 the pre-smoothing directions, deg .. 2 deg - 2 the post-smoothing directions;
  // kTermDotBufs x nterms, cleared by the restriction into the level at the start of each V-cycle
  double* tdb64 = nullptr;
  float* tdb32 = nullptr;
  uint8_t* tag = nullptr;                 // compressed stencil (level 1): material tag per node, 0 = stored
  double *pat64 = nullptr, *tmat64 = nullptr;
  float *pat32 = nullptr, *tmat32 = nullptr;
  AxisHost ax[3];                         // transfer to the next level
  TransferDev P{};
  double *b64 = nullptr, *x64 = nullptr, *r64 = nullptr, *d64 = nullptr, *t64 = nullptr, *e64 = nullptr;
  float *b32 = nullptr, *x32 = nullptr, *r32 = nullptr, *d32 = nullptr, *t32 = nullptr, *e32 = nullptr;
};

int upload_node_csr(Pool& pool, const Entries& E, int64_t nnode, Level& V) {
  if (E.size() == 0) return FEB_OK;
  std::vector<int> ptr(nnode + 1, 0), col(E.size());
  std::vector<int8_t> rr(E.size());
  std::vector<double> v(E.size());
  std::vector<float> vf(E.size());
  for (size_t e = 0; e < E.size(); ++e) ptr[E.r[e] / 3 + 1]++;
  for (int64_t i = 0; i < nnode; ++i) ptr[i + 1] += ptr[i];
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (size_t e = 0; e < E.size(); ++e) {      // a node keeps its entries in input order; duplicates add up
    int64_t node = E.r[e] / 3;
    int at = fill[node]++;
    rr[at] = (int8_t)(E.r[e] % 3); col[at] = (int)E.c[e]; v[at] = E.v[e]; vf[at] = (float)E.v[e];
  }
  FEB_TRY(pool.upload(&V.node_ptr, ptr.data(), ptr.size()));
  FEB_TRY(pool.upload(&V.ent_r, rr.data(), rr.size()));
  FEB_TRY(pool.upload(&V.ent_col, col.data(), col.size()));
  FEB_TRY(pool.upload(&V.ent_v64, v.data(), v.size()));
  FEB_TRY(pool.upload(&V.ent_v32, vf.data(), vf.size()));
  return FEB_OK;
}

// device copy of a level's terms: entries (dof, value) per term, and per node the (term, v_t at the node)
// pairs of the terms touching it
int upload_terms(Pool& pool, const Terms& T, int64_t nnode, Level& V) {
  V.nterms = (int)T.size();
  if (V.nterms == 0) return FEB_OK;
  std::vector<int> tp(T.ptr.begin(), T.ptr.end()), td(T.dof.begin(), T.dof.end());
  std::vector<float> tv32(T.val.begin(), T.val.end()), tl32(T.lam.begin(), T.lam.end());
  // pairs: one per (term, node) with the node's three components
  std::vector<int> cnt(nnode + 1, 0);
  std::vector<std::pair<int64_t, int>> pairs;   // (node, term) in term order, one per distinct node
  for (size_t t = 0; t < T.size(); ++t)
    for (int64_t e = T.ptr[t]; e < T.ptr[t + 1]; ++e)
      if (e == T.ptr[t] || T.dof[e] / 3 != T.dof[e - 1] / 3) pairs.emplace_back(T.dof[e] / 3, (int)t);
  for (const auto& pr : pairs) cnt[pr.first + 1]++;
  for (int64_t i = 0; i < nnode; ++i) cnt[i + 1] += cnt[i];
  std::vector<int> fill(cnt.begin(), cnt.end() - 1), term(pairs.size());
  std::vector<double> coef(3 * pairs.size(), 0.0);
  size_t q = 0;
  for (size_t t = 0; t < T.size(); ++t)
    for (int64_t e = T.ptr[t]; e < T.ptr[t + 1]; ++e) {
      const int64_t node = T.dof[e] / 3;
      if (e == T.ptr[t] || node != T.dof[e - 1] / 3) {
        const int at = fill[node]++;
        term[at] = (int)t;
        q = (size_t)at;
      }
      coef[3 * q + T.dof[e] % 3] = T.val[e];
    }
  std::vector<float> coef32(coef.begin(), coef.end());
  FEB_TRY(pool.upload(&V.t_ptr, tp.data(), tp.size()));
  FEB_TRY(pool.upload(&V.t_dof, td.data(), td.size()));
  FEB_TRY(pool.upload(&V.t_val64, T.val.data(), T.val.size()));
  FEB_TRY(pool.upload(&V.t_val32, tv32.data(), tv32.size()));
  FEB_TRY(pool.upload(&V.t_lam64, T.lam.data(), T.lam.size()));
  FEB_TRY(pool.upload(&V.t_lam32, tl32.data(), tl32.size()));
  FEB_TRY(pool.upload(&V.tn_ptr, cnt.data(), cnt.size()));
  FEB_TRY(pool.upload(&V.tn_term, term.data(), term.size()));
  FEB_TRY(pool.upload(&V.tn_coef64, coef.data(), coef.size()));
  FEB_TRY(pool.upload(&V.tn_coef32, coef32.data(), coef32.size()));
  FEB_TRY(pool.alloc(&V.tdot64, T.size()));
  FEB_TRY(pool.alloc(&V.tdot32, T.size()));
  FEB_TRY(pool.zeros(&V.tdb64, kTermDotBufs * T.size()));
  FEB_TRY(pool.zeros(&V.tdb32, kTermDotBufs * T.size()));
  return FEB_OK;
}

}  // namespace
}  // namespace feb

using namespace feb;

// own non-blocking stream (stream capture is impossible on the legacy default stream); ordered with the
// caller's stream by events at every entry point
// Pinned host slots for the CG state read-backs.  Page-locking host memory can take tens of milliseconds
// when the system is busy, so the slots come from blocks that are allocated once and reused by every handle
// of the process (a handle takes a slot at creation and returns it when destroyed).
namespace feb {
class PinnedSlots {
 public:
  CgState* take() {
    std::lock_guard<std::mutex> lock(mu_);
    if (free_.empty()) {
      CgState* blk = nullptr;
      if (cudaMallocHost(&blk, kBlock * sizeof(CgState)) != cudaSuccess) return nullptr;
      for (int i = kBlock - 1; i >= 0; --i) free_.push_back(blk + i);
    }
    CgState* p = free_.back();
    free_.pop_back();
    return p;
  }
  void give(CgState* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(mu_);
    free_.push_back(p);
  }

 private:
  static constexpr int kBlock = 64;
  std::mutex mu_;
  std::vector<CgState*> free_;   // blocks stay allocated until the process exits
};
static PinnedSlots g_pinned;

// Streams and events of closed handles are kept, per device, for the next handle: creating them can wait on
// the driver's resource manager, which a concurrent monitoring query (nvidia-smi, NVML) holds for milliseconds,
// so a warm process creates none.  Every event is timing-enabled.
class StreamCache {
 public:
  cudaStream_t stream() {
    const int dev = device();
    {
      std::lock_guard<std::mutex> lock(mu_);
      auto& v = streams_[dev];
      if (!v.empty()) { cudaStream_t st = v.back(); v.pop_back(); return st; }
    }
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    return st;
  }
  cudaEvent_t event() {
    const int dev = device();
    {
      std::lock_guard<std::mutex> lock(mu_);
      auto& v = events_[dev];
      if (!v.empty()) { cudaEvent_t e = v.back(); v.pop_back(); return e; }
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
  }
  // a stream is given back idle (the caller synchronised it)
  void give(cudaStream_t st) {
    if (!st) return;
    std::lock_guard<std::mutex> lock(mu_);
    streams_[device()].push_back(st);
  }
  void give(cudaEvent_t e) {
    if (!e) return;
    std::lock_guard<std::mutex> lock(mu_);
    events_[device()].push_back(e);
  }

 private:
  static int device() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) { cudaGetLastError(); d = 0; }
    return d;
  }
  std::mutex mu_;
  std::map<int, std::vector<cudaStream_t>> streams_;   // kept until the process exits
  std::map<int, std::vector<cudaEvent_t>> events_;
};
static StreamCache g_streams;
}  // namespace feb

static cudaStream_t make_stream() { return feb::g_streams.stream(); }

struct FebHandle {
  explicit FebHandle(cudaStream_t caller_) : caller(caller_), s(make_stream()), pool(s) {
    ev_sync = g_streams.event();
  }
  cudaStream_t caller;
  cudaStream_t s;
  Pool pool;
  cudaEvent_t ev_sync = nullptr;
  // work on s after everything queued so far on the caller's stream
  int sync_in() {
    FEB_CUDA(cudaEventRecord(ev_sync, caller));
    FEB_CUDA(cudaStreamWaitEvent(s, ev_sync, 0));
    return FEB_OK;
  }
  // the caller's stream continues after everything queued on s
  int sync_out() {
    FEB_CUDA(cudaEventRecord(ev_sync, s));
    FEB_CUDA(cudaStreamWaitEvent(caller, ev_sync, 0));
    return FEB_OK;
  }
  FebOptions opt{};
  int mode = MAT_ISO_SRI;
  int nx = 0, ny = 0, nz = 0;
  std::vector<double> xe, ye, ze;
  int64_t nnode = 0, ntotal = 0, ndof = 0;
  FineView<double> F64{};
  FineView<float> F32{};
  bool tc_ok = false;                     // FP32 K.u may run on the tensor cores (equal cubic cells, ISO model)
  int* tc_status = nullptr;
  int* orig_copy = nullptr;
  std::vector<int64_t> orig_copy_h;
  double *xe_d = nullptr, *ye_d = nullptr, *ze_d = nullptr;
  // penalties and local extra entries of level 0, for the level-1 Galerkin product
  int npen = 0;
  int nlocal = 0;
  int *loc_r = nullptr, *loc_c = nullptr;
  double* loc_v = nullptr;
  double* mat_all = nullptr;
  // level-1 stencil summed directly from the fine cells, launched on a side stream while the host prepares the
  // penalties and extra entries (A1_early, ready at A1_ev; basis: its sub-cell matrices)
  double* A1_early = nullptr;
  double* A1_basis = nullptr;
  cudaEvent_t A1_ev = nullptr;
  std::vector<Level> L;
  int coarsest = 0;
  // dense coarsest level
  int nd = 0;
  double *Minv = nullptr;
  int *klist = nullptr, *cmap = nullptr;
  // scalars
  LevelParams* lp = nullptr;
  CgState* st = nullptr;      // outer CG
  CgState* sti = nullptr;     // inner CG (refinement)
  double* partials = nullptr;
  unsigned int* ctr = nullptr;   // arrival counter of the last-block reductions (zero between launches)
  double* sc = nullptr;       // refinement scaling
  int* status = nullptr;
  CgState* st_h = nullptr;    // pinned
  // CG vectors
  double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *fb = nullptr;
  float *xf = nullptr, *rf = nullptr, *zf = nullptr, *pf = nullptr, *qf = nullptr;
  // rigid modes
  bool has_rigid = false;
  RigidView Z{};
  double *Einv = nullptr, *zpart = nullptr, *zr = nullptr, *zcoef = nullptr;
  // graphs
  cudaGraphExec_t g_outer = nullptr, g_inner = nullptr;
  int g_outer_nodes = 0, g_inner_nodes = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t tev0 = nullptr, tev1 = nullptr;   // the autotuner's timings (ev0 marks the set-up's start)
  int tune_events() {
    if (!tev0 && !(tev0 = g_streams.event())) { set_last_error("cudaEventCreate"); return FEB_ERR_CUDA; }
    if (!tev1 && !(tev1 = g_streams.event())) { set_last_error("cudaEventCreate"); return FEB_ERR_CUDA; }
    return FEB_OK;
  }
  KuConfig ku32{}, ku64{};   // launch shapes of the fine K.u (autotuned per grid shape)
  // paired-row level-0 kernels (fine_pair.cu): used when every regular cell's material fits the id table
  bool pair_ok = false;
  PairView<float> P32{};
  PairView<double> P64{};
  PairConfig pc32{}, pc64{};
  float* D6_32 = nullptr;    // level-0 symmetric block-Jacobi inverse [6][ntotal]
  double* D6_64 = nullptr;
  static constexpr int kStages = 10;
  cudaEvent_t stage_ev[kStages + 1] = {};
  int stage_n = 0;
  double stage_ms[kStages] = {};
  void stage_mark() {   // event after each set-up stage (device time between consecutive marks)
    if (stage_n <= kStages) cudaEventRecord(stage_ev[stage_n++], s);
  }
  double t_setup_ms = 0.0;
  double t_pre_ms = 0.0;    // host time of feb_create before the device-timed set-up (pool reservation, handle)
  int launches = 0;

  // side streams of set-up work that runs per level (power iterations), with their join events
  static constexpr int kAux = kMaxLevels;
  cudaStream_t aux[kAux] = {};
  cudaEvent_t aux_ev[kAux] = {};

  // Set-up work still running when feb_create returns: the power iterations (aux streams) and the dense
  // coarsest level with its inverse (dense_s).  The caller's next steps (rigid groups, loads, a start value)
  // overlap them on the device; settle() joins them into s before anything reads their results.
  bool pending = false;
  int coarse_fail = 0;                    // the coarsest-level matrix was not positive definite
  cudaStream_t dense_s = nullptr;
  cudaEvent_t dense_ev = nullptr;
  int* dense_st = nullptr;                // device status of the inverse, copied to dense_st_h (pinned)
  CgState* dense_st_h = nullptr;
  std::vector<void*> deferred_free;       // buffers the deferred work reads, freed on s once joined

  int coarse_error() {
    set_last_error("coarsest-level matrix (%d dofs) is not positive definite", nd);
    return FEB_ERR_COARSE;
  }
  // joins the deferred set-up into s, frees what only it needed, completes the set-up times and reports a
  // failed coarsest-level inverse (then and on every later call)
  int settle() {
    if (!pending) return coarse_fail ? coarse_error() : FEB_OK;
    pending = false;
    for (int k = 0; k < coarsest; ++k) FEB_CUDA(cudaStreamWaitEvent(s, aux_ev[k], 0));
    FEB_CUDA(cudaStreamWaitEvent(s, dense_ev, 0));
    for (void* p : deferred_free) pool.free(p);
    deferred_free.clear();
    FEB_CUDA(cudaEventSynchronize(dense_ev));
    for (int k = 0; k < coarsest; ++k) FEB_CUDA(cudaEventSynchronize(aux_ev[k]));
    // stage 6: from the end of the enqueue to the end of the slowest deferred chain; the set-up's span
    float t = 0.f, tail = 0.f, span = (float)t_setup_ms;
    auto upto = [&](cudaEvent_t e) {
      if (cudaEventElapsedTime(&t, stage_ev[6], e) == cudaSuccess) tail = std::max(tail, t);
      if (cudaEventElapsedTime(&t, ev0, e) == cudaSuccess) span = std::max(span, t);
    };
    upto(dense_ev);
    for (int k = 0; k < coarsest; ++k) upto(aux_ev[k]);
    cudaGetLastError();
    stage_ms[6] = tail;
    t_setup_ms = span;
    coarse_fail = *reinterpret_cast<volatile int*>(dense_st_h) != 0;
    return coarse_fail ? coarse_error() : FEB_OK;
  }

  // the level-0 products share their sparse-part accumulators with the level-0 power iteration: a product on
  // s waits (on the device) for that chain while it may still run
  int wait_fine() {
    if (pending && coarsest > 0) FEB_CUDA(cudaStreamWaitEvent(s, aux_ev[0], 0));
    return FEB_OK;
  }

  // the rigid-mode coefficients' stream (set with the rigid groups) and its fork / join events
  cudaStream_t rs = nullptr;
  cudaEvent_t rs_fork = nullptr, rs_join = nullptr;

  ~FebHandle() {
    if (rs) { cudaStreamSynchronize(rs); g_streams.give(rs); }
    g_streams.give(rs_fork);
    g_streams.give(rs_join);
    if (dense_s) { cudaStreamSynchronize(dense_s); g_streams.give(dense_s); }
    g_streams.give(dense_ev);
    g_pinned.give(dense_st_h);
    for (int i = 0; i < kAux; ++i) {
      if (aux[i]) { cudaStreamSynchronize(aux[i]); g_streams.give(aux[i]); }
      g_streams.give(aux_ev[i]);
    }
    g_streams.give(A1_ev);
    if (g_outer) cudaGraphExecDestroy(g_outer);
    if (g_inner) cudaGraphExecDestroy(g_inner);
    g_pinned.give(st_h);
    g_streams.give(ev0);
    g_streams.give(tev0);
    g_streams.give(tev1);
    g_streams.give(ev1);
    pool.release();
    cudaStreamSynchronize(s);
    g_streams.give(ev_sync);
    for (auto& e : stage_ev) g_streams.give(e);
    g_streams.give(s);
  }

  // ---------------------------------------------------------------------------------------------- operators
  template <typename T>
  const FineView<T>& fine() const;

  template <typename T> const PairView<T>& pview() const;
  template <typename T> const T* dinv6() const;
  template <typename T>
  PairConfig pcfg() const { return std::is_same<T, double>::value ? pc64 : pc32; }
  // the paired kernel serves precision T (FEB_KU_TC=1 keeps FP32 products on the tensor-core kernel)
  template <typename T>
  bool pair_on() const { return pair_ok && (std::is_same<T, double>::value || !(tc_ok && ku32.tc)); }
  template <typename T>
  void pair_run(const T* u, T* y, const SmoothArgs<T>* S, const int* skip) {
    switch (mode) {
      case MAT_ISO_SRI: launch_fine_pair<T, MAT_ISO_SRI>(pview<T>(), fine<T>(), u, y, S, skip, pcfg<T>(), s); break;
      case MAT_ISO_FULL: launch_fine_pair<T, MAT_ISO_FULL>(pview<T>(), fine<T>(), u, y, S, skip, pcfg<T>(), s); break;
      default: launch_fine_pair<T, MAT_ORTHO>(pview<T>(), fine<T>(), u, y, S, skip, pcfg<T>(), s); break;
    }
  }

  template <typename T>
  void apply(int l, const T* u, T* y, const int* skip) {
    if (l == 0 && pair_on<T>()) {
      pair_run<T>(u, y, nullptr, skip);
      return;
    }
    if (l == 0) {
      const FineView<T>& F = fine<T>();
      const KuConfig cfg = std::is_same<T, double>::value ? ku64 : ku32;
      switch (mode) {
        case MAT_ISO_SRI: launch_fine_apply<T, MAT_ISO_SRI>(F, u, y, skip, cfg, s); break;
        case MAT_ISO_FULL: launch_fine_apply<T, MAT_ISO_FULL>(F, u, y, skip, cfg, s); break;
        default: launch_fine_apply<T, MAT_ORTHO>(F, u, y, skip, cfg, s); break;
      }
    } else {
      launch_sym<T>(symview<T>(L[l]), EPI_APPLY, u, y, nullptr, nullptr, nullptr, nullptr, nullptr, 0, skip, s);
    }
  }
  template <typename T>
  SymView<T> symview(const Level& V) const {
    SymView<T> S;
    S.nx = V.nx; S.ny = V.ny; S.nz = V.nz; S.n = V.nnode;
    S.nxp = sym_nxp(V.nx); S.np = sym_np(V.nx, V.ny, V.nz);
    S.slots = opt.level_kernel & 3;
    S.S = symS<T>(V);
    if constexpr (std::is_same<T, float>::value) { S.Sh = V.S16; S.hscale = V.hscale; }
    S.node_ptr = V.node_ptr; S.ent_r = V.ent_r; S.ent_col = V.ent_col; S.ent_v = entv<T>(V);
    S.tn_ptr = V.nterms ? V.tn_ptr : nullptr; S.tn_term = V.tn_term; S.tn_coef = tcoef<T>(V);
    S.t_ptr = V.t_ptr; S.t_dof = V.t_dof; S.t_val = tval<T>(V); S.t_lam = tlam<T>(V);
    S.nterms = V.nterms;
    if constexpr (std::is_same<T, double>::value) S.tdot = V.tdot64; else S.tdot = V.tdot32;
    S.Dinv = dinv<T>(V);
    if (V.tag) {
      S.tag = V.tag;
      if constexpr (std::is_same<T, double>::value) { S.pat = V.pat64; S.tmat = V.tmat64; }
      else { S.pat = V.pat32; S.tmat = V.tmat32; }
    }
    return S;
  }
  template <typename T> static const T* symS(const Level& V);
  template <typename T> static const T* entv(const Level& V);
  template <typename T> static const T* tcoef(const Level& V);
  template <typename T> static const T* tval(const Level& V);
  template <typename T> static const T* tlam(const Level& V);
  template <typename T> static T* ve(Level& V);
  template <typename T> static const T* dinv(const Level& V);
  template <typename T> static T* vb(Level& V);
  template <typename T> static T* vx(Level& V);
  template <typename T> static T* vr(Level& V);
  template <typename T> static T* vd(Level& V);
  template <typename T> static T* vt(Level& V);
  template <typename T> T* tdb(Level& V) const {
    if (!V.nterms || (opt.level_kernel & 4)) return nullptr;   // bit 2: a dot pass before every product instead
    if constexpr (std::is_same<T, double>::value) return V.tdb64; else return V.tdb32;
  }
  // the V-cycle's term-dot accumulation at level V into dot buffers a, b (either may be null)
  template <typename T>
  static TermAcc<T> term_acc(Level& V, T* a, T* b) {
    TermAcc<T> A;
    if (!V.nterms || (!a && !b)) return A;
    A.tn_ptr = V.tn_ptr; A.tn_term = V.tn_term; A.tn_coef = tcoef<T>(V); A.t_lam = tlam<T>(V);
    A.dot_a = a; A.dot_b = b;
    return A;
  }

  // ---------------------------------------------------------------------------------------------- V-cycle
  template <typename T>
  void smooth(int l, const T* b, T* x, bool zero_start, const int* skip) {
    if (l > 0) {   // stencil level: residual and Chebyshev steps fused with the stencil product
      Level& V = L[l];
      const SymView<T> SV = symview<T>(V);
      T *r = vr<T>(V), *d = vd<T>(V), *e = ve<T>(V);
      const T* D = dinv<T>(V);
      // term dots of each product's input come from the kernel that wrote it (no dot pass): the iterate's
      // (buffer 0) while pre-smoothing, whose result the residual reads; each step's direction but the last's
      T* B = tdb<T>(V);
      const int deg = opt.cheb_degree, base = zero_start ? 1 : deg;
      auto buf = [&](int i) { return B ? B + (size_t)i * V.nterms : nullptr; };
      T* tdx = buf(0);
      if (zero_start) {
        launch_cheb_first<T>(b, r, d, x, D, lp + l, V.ntotal, skip, s,
                             term_acc<T>(V, deg > 1 ? buf(base) : nullptr, tdx));
      } else {
        launch_sym<T>(SV, EPI_RESID, x, nullptr, b, r, nullptr, nullptr, nullptr, 0, skip, s, tdx);
        launch_cheb_from_r<T>(r, d, x, D, lp + l, V.ntotal, skip, s,
                              term_acc<T>(V, deg > 1 ? buf(base) : nullptr, nullptr));
      }
      for (int k = 0; k + 1 < deg; ++k) {
        const bool last = k + 2 == deg;
        launch_sym<T>(SV, EPI_CHEB, d, nullptr, nullptr, r, e, x, lp + l, k, skip, s, buf(base + k),
                      term_acc<T>(V, last ? nullptr : buf(base + k + 1), zero_start ? tdx : nullptr));
        std::swap(d, e);
      }
      return;
    }
    Level& V = L[l];
    const int64_t nn = V.ntotal;
    T *r = vr<T>(V), *d = vd<T>(V), *t = vt<T>(V);
    const T* D = dinv<T>(V);
    if (zero_start) {
      launch_cheb_first<T>(b, r, d, x, D, lp + l, nn, skip, s);
    } else {
      apply<T>(l, x, t, skip);
      launch_cheb_init<T>(b, t, r, d, x, D, lp + l, nn, skip, s);
    }
    for (int k = 0; k + 1 < opt.cheb_degree; ++k) {
      apply<T>(l, d, t, skip);
      launch_cheb_step<T>(t, r, d, x, D, lp + l, k, nn, skip, s);
    }
  }

  // Level-0 V-cycle leg with the smoother fused into the paired K.u (same arithmetic as smooth() +
  // residual + transfers): pre-smoothing from zero keeps x = d0 + d1 + ... and the residual of the smoothed
  // iterate is r - K d_last; post-smoothing starts from xs and writes the result into x.
  // x64 (optional): the last post-smoothing step writes the result there in FP64 instead of into x
  template <typename T>
  void vcycle0_pair(const T* b, T* x, const int* skip, double* x64 = nullptr) {
    Level& V = L[0];
    Level& C = L[1];
    T *r = vr<T>(V), *d = vd<T>(V), *e = ve<T>(V), *xs = vt<T>(V);
    const int deg = std::max(1, opt.cheb_degree);
    launch_cheb_first6<T>(b, dinv6<T>(), lp, d, deg == 1 ? xs : nullptr, ntotal, skip, s);
    for (int k = 1; k < deg; ++k) {
      SmoothArgs<T> A;
      A.r_in = (k == 1) ? b : r; A.r_out = r; A.x_in = (k == 1) ? d : xs; A.x_out = xs; A.d_out = e; A.lp = lp;
      A.k = k - 1;
      pair_run<T>(d, nullptr, &A, skip);
      std::swap(d, e);
    }
    {
      SmoothArgs<T> A;
      A.r_in = (deg == 1) ? b : r; A.r_out = r;
      pair_run<T>(d, nullptr, &A, skip);
    }
    launch_restrict<T>(V.P, V.nx, V.ny, V.nz, V.nnode, V.ntotal, orig_copy, r, vb<T>(C), skip, s, tdb<T>(C),
                       kTermDotBufs * C.nterms);
    vcycle<T>(1, vb<T>(C), vx<T>(C), skip);
    launch_prolong_add<T>(V.P, V.nx, V.ny, V.nz, V.nnode, V.ntotal, orig_copy, V.used, vx<T>(C), xs, skip, s);
    {
      SmoothArgs<T> A;
      A.r_in = b; A.r_out = deg > 1 ? r : nullptr; A.x_in = xs; A.d_out = deg > 1 ? d : nullptr;
      if (deg == 1 && x64) A.x_out64 = x64; else A.x_out = x;
      A.lp = lp; A.k = -1;
      pair_run<T>(xs, nullptr, &A, skip);
    }
    for (int k = 1; k < deg; ++k) {
      const bool last = (k == deg - 1);
      SmoothArgs<T> A;
      A.r_in = r; A.r_out = last ? nullptr : r; A.x_in = x; A.d_out = last ? nullptr : e; A.lp = lp;
      if (last && x64) A.x_out64 = x64; else A.x_out = x;
      A.k = k - 1;
      pair_run<T>(d, nullptr, &A, skip);
      std::swap(d, e);
    }
  }

  template <typename T>
  void vcycle(int l, const T* b, T* x, const int* skip) {
    if (l == 0 && coarsest > 0 && pair_on<T>()) {
      vcycle0_pair<T>(b, x, skip);
      return;
    }
    if (l == coarsest) {
      Level& V = L[l];
      launch_dense_solve<T>(Minv, nd, klist, cmap, V.ntotal, b, x, skip, s);
      return;
    }
    Level& V = L[l];
    Level& C = L[l + 1];
    smooth<T>(l, b, x, true, skip);
    T *t = vt<T>(V), *r = vr<T>(V);
    T* tdx = tdb<T>(V);   // level l's iterate dots (buffer 0; null at level 0 and on levels without terms)
    if (l > 0) {
      launch_sym<T>(symview<T>(V), EPI_RESID, x, nullptr, b, r, nullptr, nullptr, nullptr, 0, skip, s, tdx);
    } else {
      apply<T>(l, x, t, skip);
      launch_residual<T>(b, t, r, 3 * V.ntotal, skip, s);
    }
    launch_restrict<T>(V.P, V.nx, V.ny, V.nz, V.nnode, V.ntotal, orig_copy, r, vb<T>(C), skip, s, tdb<T>(C),
                       kTermDotBufs * C.nterms);
    vcycle<T>(l + 1, vb<T>(C), vx<T>(C), skip);
    launch_prolong_add<T>(V.P, V.nx, V.ny, V.nz, V.nnode, V.ntotal, orig_copy, V.used, vx<T>(C), x, skip, s,
                          term_acc<T>(V, nullptr, tdx));
    smooth<T>(l, b, x, false, skip);
  }

  // z = M r for the CG of precision T (FP64 CG with an FP64 or FP32 V-cycle, FP32 CG with FP32); rf_ready:
  // the FP32 copy of r (rf) was written by the CG update already
  template <typename T>
  void precondition(const T* r_, T* z_, const int* skip, bool rf_ready = false) {
    const int64_t n = 3 * ntotal;
    if (has_rigid && rs) {   // Einv Z^T r reads r only: it runs on the rigid-mode stream beside the V-cycle
      cudaEventRecord(rs_fork, s);
      cudaStreamWaitEvent(rs, rs_fork, 0);
      launch_rigid_coef<T>(Z, r_, zpart, zr, zcoef, Einv, skip, rs, ctr + 1);
      cudaEventRecord(rs_join, rs);
    }
    if constexpr (std::is_same<T, double>::value) {
      if (opt.precision == FEB_PREC_FP64) {
        vcycle<double>(0, r_, z_, skip);
      } else {
        if (!rf_ready) launch_convert<double, float>(r_, rf, n, skip, s);
        if (coarsest > 0 && pair_on<float>()) {
          vcycle0_pair<float>(rf, zf, skip, z_);   // its last smoothing step writes z in FP64
        } else {
          vcycle<float>(0, rf, zf, skip);
          launch_convert<float, double>(zf, z_, n, skip, s);
        }
      }
    } else {
      vcycle<float>(0, r_, z_, skip);
    }
    if (has_rigid && rs) {
      cudaStreamWaitEvent(s, rs_join, 0);
      launch_rigid_scatter<T>(Z, zcoef, z_, skip, s);
    } else if (has_rigid) {
      launch_rigid_apply<T>(Z, r_, z_, zpart, zr, zcoef, Einv, skip, s, ctr + 1);
    }
  }

  // one CG iteration (SciPy order: z = M r, beta, p, q = A p, alpha, x, r, convergence)
  template <typename T>
  void cg_body(CgState* S, T* x_, T* r_, T* z_, T* p_, T* q_) {
    const int* skip = &S->done;
    const int64_t n = 3 * ntotal;
    // the mixed precision's FP32 copy of r is written by the x/r update (and by cg_start before the loop)
    const bool mixed = std::is_same<T, double>::value && opt.precision != FEB_PREC_FP64;
    precondition<T>(r_, z_, skip, mixed);
    launch_dot_finalize<T, T>(FIN_RZ, r_, z_, n, partials, ctr, S, skip, s);
    launch_update_p<T>(z_, p_, S, n, skip, s);
    apply<T>(0, p_, q_, skip);
    launch_dot_finalize<T, T>(FIN_ALPHA, p_, q_, n, partials, ctr, S, skip, s);
    launch_update_xr_conv<T>(p_, q_, x_, r_, mixed ? rf : nullptr, S, n, partials, ctr, skip, s);
  }

  // one CG iteration captured as a graph; with use_graphs == 2 the iteration is the body of a device-side
  // while loop (conditional graph node): the whole CG then runs as one graph launch
  int capture(CgState* S, bool inner, cudaGraphExec_t* exec, int* nodes) {
    if (*exec) return FEB_OK;
    struct Capturing {
      Capturing() { g_capturing = true; }
      ~Capturing() { g_capturing = false; }
    } capturing;
    cudaGraph_t g = nullptr;
    if (opt.use_graphs >= 2) {
      FEB_CUDA(cudaGraphCreate(&g, 0));
      cudaGraphConditionalHandle cond;
      FEB_CUDA(cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = cond;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t node;
      FEB_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      FEB_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
      if (inner) cg_body<float>(S, xf, rf, zf, pf, qf);
      else cg_body<double>(S, x, r, z, p, q);
      launch_set_condition(cond, S, s);
      FEB_CUDA(cudaStreamEndCapture(s, &body));
      size_t nn = 0;
      FEB_CUDA(cudaGraphGetNodes(body, nullptr, &nn));
      *nodes = (int)nn;
    } else {
      FEB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      if (inner) cg_body<float>(S, xf, rf, zf, pf, qf);
      else cg_body<double>(S, x, r, z, p, q);
      FEB_CUDA(cudaStreamEndCapture(s, &g));
      size_t nn = 0;
      FEB_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
      *nodes = (int)nn;
    }
    FEB_CUDA(cudaGraphInstantiate(exec, g, 0));
    FEB_CUDA(cudaGraphDestroy(g));
    return FEB_OK;
  }

  // the CG iteration graph, captured ahead of the first solve (feb_set_rigid_groups does it beside its products)
  int prepare_graphs() {
    if (!opt.use_graphs || coarsest < 0) return FEB_OK;
    return opt.precision == FEB_PREC_REFINE ? capture(sti, true, &g_inner, &g_inner_nodes)
                                            : capture(st, false, &g_outer, &g_outer_nodes);
  }

  // runs CG iterations until S->done; returns the final host copy of the state
  int run_cg(CgState* S, bool inner, CgState& out) {
    cudaGraphExec_t* ex = inner ? &g_inner : &g_outer;
    int* nn = inner ? &g_inner_nodes : &g_outer_nodes;
    if (opt.use_graphs) FEB_TRY(capture(S, inner, ex, nn));
    if (opt.use_graphs >= 2) {   // device-side loop: one launch, one synchronisation
      FEB_CUDA(cudaGraphLaunch(*ex, s));
      FEB_CUDA(cudaMemcpyAsync(st_h, S, sizeof(CgState), cudaMemcpyDeviceToHost, s));
      FEB_CUDA(cudaStreamSynchronize(s));
      const int iters = st_h->it > 0 ? st_h->it : 1;
      launches += iters * (*nn);
      note_launch(iters * (*nn));
      out = *st_h;
      return FEB_OK;
    }
    const int every = std::max(1, opt.check_every);
    for (int guard = 0; guard < 1000000; ++guard) {
      FEB_CUDA(cudaMemcpyAsync(st_h, S, sizeof(CgState), cudaMemcpyDeviceToHost, s));
      FEB_CUDA(cudaStreamSynchronize(s));
      if (st_h->done) break;
      for (int k = 0; k < every; ++k) {
        if (opt.use_graphs) {
          FEB_CUDA(cudaGraphLaunch(*ex, s));
          launches += *nn;
          note_launch(*nn);
        } else {
          if (inner) cg_body<float>(S, xf, rf, zf, pf, qf);
          else cg_body<double>(S, x, r, z, p, q);
        }
      }
    }
    FEB_CUDA(cudaGetLastError());
    out = *st_h;
    return FEB_OK;
  }

  // CG on K x = b in precision T from x (x0 given or zero); thr = tol ||b||
  template <typename T>
  int cg_start(CgState* S, const T* b, T* x_, T* r_, bool has_x0, double thr2, int maxiter) {
    const int64_t n = 3 * ntotal;
    CgState init{};
    init.thr2 = thr2;
    init.maxiter = maxiter;
    FEB_CUDA(cudaMemcpyAsync(S, &init, sizeof(CgState), cudaMemcpyHostToDevice, s));
    if (has_x0) {
      T* q_ = std::is_same<T, double>::value ? (T*)q : (T*)qf;
      apply<T>(0, x_, q_, nullptr);
      launch_residual<T>(b, q_, r_, n, nullptr, s);
    } else {
      FEB_CUDA(cudaMemsetAsync(x_, 0, n * sizeof(T), s));
      FEB_CUDA(cudaMemcpyAsync(r_, b, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
    }
    launch_dot_partial<T, T>(r_, r_, n, partials, nullptr, s);
    launch_finalize(FIN_INIT, partials, S, nullptr, 0, nullptr, s);
    launches += has_x0 ? 6 : 2;
    if (std::is_same<T, double>::value && opt.precision != FEB_PREC_FP64) {   // FP32 copy for the first V-cycle
      launch_convert<double, float>((const double*)r_, rf, n, nullptr, s);
      launches += 1;
    }
    return FEB_OK;
  }

  double read_dot(const double* a, const double* b, int64_t n, int* st) {
    launch_dot_partial<double, double>(a, b, n, partials, nullptr, s);
    std::vector<double> h(kRedBlocks);
    cudaError_t e = cudaMemcpyAsync(h.data(), partials, kRedBlocks * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_last_error("read_dot: %s", cudaGetErrorString(e)); *st = FEB_ERR_CUDA; return 0.0; }
    double acc = 0.0;
    for (double v : h) acc += v;
    return acc;
  }
};

template <> const PairView<double>& FebHandle::pview<double>() const { return P64; }
template <> const PairView<float>& FebHandle::pview<float>() const { return P32; }
template <> const double* FebHandle::dinv6<double>() const { return D6_64; }
template <> const float* FebHandle::dinv6<float>() const { return D6_32; }
template <> const FineView<double>& FebHandle::fine<double>() const { return F64; }
template <> const FineView<float>& FebHandle::fine<float>() const { return F32; }
template <> const double* FebHandle::dinv<double>(const Level& V) { return V.Dinv64; }
template <> const float* FebHandle::dinv<float>(const Level& V) { return V.Dinv32; }
template <> double* FebHandle::vb<double>(Level& V) { return V.b64; }
template <> float* FebHandle::vb<float>(Level& V) { return V.b32; }
template <> double* FebHandle::vx<double>(Level& V) { return V.x64; }
template <> float* FebHandle::vx<float>(Level& V) { return V.x32; }
template <> double* FebHandle::vr<double>(Level& V) { return V.r64; }
template <> float* FebHandle::vr<float>(Level& V) { return V.r32; }
template <> double* FebHandle::vd<double>(Level& V) { return V.d64; }
template <> float* FebHandle::vd<float>(Level& V) { return V.d32; }
template <> double* FebHandle::vt<double>(Level& V) { return V.t64; }
template <> float* FebHandle::vt<float>(Level& V) { return V.t32; }
template <> double* FebHandle::ve<double>(Level& V) { return V.e64; }
template <> float* FebHandle::ve<float>(Level& V) { return V.e32; }
template <> const double* FebHandle::symS<double>(const Level& V) { return V.S64; }
template <> const float* FebHandle::symS<float>(const Level& V) { return V.S32; }
template <> const double* FebHandle::entv<double>(const Level& V) { return V.ent_v64; }
template <> const double* FebHandle::tcoef<double>(const Level& V) { return V.tn_coef64; }
template <> const float* FebHandle::tcoef<float>(const Level& V) { return V.tn_coef32; }
template <> const double* FebHandle::tval<double>(const Level& V) { return V.t_val64; }
template <> const float* FebHandle::tval<float>(const Level& V) { return V.t_val32; }
template <> const double* FebHandle::tlam<double>(const Level& V) { return V.t_lam64; }
template <> const float* FebHandle::tlam<float>(const Level& V) { return V.t_lam32; }
template <> const float* FebHandle::entv<float>(const Level& V) { return V.ent_v32; }


namespace feb {
namespace {

__global__ void k_count(const uint8_t* __restrict__ m, int64_t n, unsigned long long* __restrict__ out) {
  unsigned long long c = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    c += m[i] ? 1ull : 0ull;
  c = block_sum(c);
  if (threadIdx.x == 0) atomicAdd(out, c);
}

int count_mask(FebHandle* h, const uint8_t* m, int64_t n, int64_t* out) {
  unsigned long long* d = nullptr;
  FEB_TRY(h->pool.zeros(&d, 1));
  k_count<<<std::min<int64_t>(div_up(n, kThreads), 4 * kSmCount), kThreads, 0, h->s>>>(m, n, d); note_launch();
  unsigned long long v = 0;
  FEB_CUDA(cudaMemcpyAsync(&v, d, sizeof(v), cudaMemcpyDeviceToHost, h->s));
  FEB_CUDA(cudaStreamSynchronize(h->s));
  h->pool.free(d);
  *out = (int64_t)v;
  return FEB_OK;
}

template <typename T>
int level_vectors(Pool& pool, Level& V, bool f64, bool f32) {
  size_t n = 3 * (size_t)V.ntotal;
  if (f64) {
    FEB_TRY(pool.zeros(&V.b64, n)); FEB_TRY(pool.zeros(&V.x64, n)); FEB_TRY(pool.zeros(&V.r64, n));
    FEB_TRY(pool.zeros(&V.d64, n)); FEB_TRY(pool.zeros(&V.t64, n)); FEB_TRY(pool.zeros(&V.e64, n));
  }
  if (f32) {
    FEB_TRY(pool.zeros(&V.b32, n)); FEB_TRY(pool.zeros(&V.x32, n)); FEB_TRY(pool.zeros(&V.r32, n));
    FEB_TRY(pool.zeros(&V.d32, n)); FEB_TRY(pool.zeros(&V.t32, n)); FEB_TRY(pool.zeros(&V.e32, n));
  }
  return FEB_OK;
}

int upload_transfer(Pool& pool, Level& V) {
  for (int d = 0; d < 3; ++d) {
    AxisHost& A = V.ax[d];
    AxisDev& D = V.P.ax[d];
    D.nf = A.nf; D.nc = A.nc;
    int *ca, *cb, *cidx, *ivf, *ivc;
    double *wa, *wb;
    FEB_TRY(pool.upload(&ca, A.ca.data(), A.ca.size()));
    FEB_TRY(pool.upload(&cb, A.cb.data(), A.cb.size()));
    FEB_TRY(pool.upload(&wa, A.wa.data(), A.wa.size()));
    FEB_TRY(pool.upload(&wb, A.wb.data(), A.wb.size()));
    FEB_TRY(pool.upload(&cidx, A.cidx.data(), A.cidx.size()));
    std::vector<int> f(A.iv_first), c(A.iv_count);
    if (f.empty()) { f.push_back(0); c.push_back(0); }
    FEB_TRY(pool.upload(&ivf, f.data(), f.size()));
    FEB_TRY(pool.upload(&ivc, c.data(), c.size()));
    D.ca = ca; D.cb = cb; D.wa = wa; D.wb = wb; D.cidx = cidx; D.iv_first = ivf; D.iv_count = ivc;
  }
  // even coarsening on every axis: 2 nc - 1 fine nodes, odd fine nodes halfway between their coarse neighbours
  bool even = true;
  for (int d = 0; d < 3 && even; ++d) {
    const AxisHost& A = V.ax[d];
    even = A.nf == 2 * A.nc - 1;
    for (int i = 0; i < A.nf && even; ++i) {
      if (i % 2 == 0) even = A.ca[i] == i / 2 && A.wa[i] == 1.0 && (A.wb[i] == 0.0 || A.cb[i] == A.ca[i]);
      else even = A.ca[i] == i / 2 && A.cb[i] == i / 2 + 1 && std::fabs(A.wa[i] - 0.5) < 1e-12 &&
                  std::fabs(A.wb[i] - 0.5) < 1e-12;
    }
  }
  V.P.even = even ? 1 : 0;
  return FEB_OK;
}

// the split copies' restriction as a gather per coarse node (even coarsening): copy c sits at fine grid
// position orig_copy[c] and restricts with the weights of that position
int upload_copy_gather(Pool& pool, Level& V, const std::vector<int64_t>& orig_copy) {
  if (!V.P.even || orig_copy.empty()) return FEB_OK;
  const int fnx = V.nx, fny = V.ny, cnx = V.ax[0].nc, cny = V.ax[1].nc, cnz = V.ax[2].nc;
  const int64_t nc = (int64_t)cnx * cny * cnz;
  std::vector<int> cnt(nc + 1, 0);
  auto each = [&](int64_t o, auto&& f) {
    const int pi = int(o % fnx), pj = int((o / fnx) % fny), pk = int(o / ((int64_t)fnx * fny));
    const int ni = (pi & 1) + 1, nj = (pj & 1) + 1, nk = (pk & 1) + 1;
    const double w = (ni == 2 ? 0.5 : 1.0) * (nj == 2 ? 0.5 : 1.0) * (nk == 2 ? 0.5 : 1.0);
    for (int c = 0; c < nk; ++c)
      for (int b = 0; b < nj; ++b)
        for (int a = 0; a < ni; ++a) f((pi >> 1) + a + (int64_t)cnx * ((pj >> 1) + b + (int64_t)cny * ((pk >> 1) + c)), w);
  };
  for (size_t c = 0; c < orig_copy.size(); ++c) each(orig_copy[c], [&](int64_t J, double) { cnt[J + 1]++; });
  for (int64_t J = 0; J < nc; ++J) cnt[J + 1] += cnt[J];
  std::vector<int> fill(cnt.begin(), cnt.end() - 1), copy(cnt[nc]);
  std::vector<double> w(cnt[nc]);
  for (size_t c = 0; c < orig_copy.size(); ++c)      // ascending copy index within each coarse node
    each(orig_copy[c], [&](int64_t J, double wt) { const int at = fill[J]++; copy[at] = (int)c; w[at] = wt; });
  int *ptr, *cp;
  double* wd;
  FEB_TRY(pool.upload(&ptr, cnt.data(), cnt.size()));
  FEB_TRY(pool.upload(&cp, copy.data(), copy.size()));
  FEB_TRY(pool.upload(&wd, w.data(), w.size()));
  V.P.cp_ptr = ptr; V.P.cp_copy = cp; V.P.cp_w = wd;
  return FEB_OK;
}

// 12 power steps for lambda_max(Dinv A) (fe/gmg.py:47-59) and the Chebyshev coefficients, in precision T.
// (on h->s, with the reduction scratch `part`)
template <typename T>
int power_iteration(FebHandle* h, int l, double* part, unsigned int* pctr) {
  Level& V = h->L[l];
  const int64_t n = 3 * V.ntotal;
  T *x = FebHandle::vx<T>(V), *t = FebHandle::vt<T>(V), *d = FebHandle::vd<T>(V);
  launch_random_start<T>(x, V.used, V.ntotal, h->opt.seed + 7919ull * (uint64_t)l, h->s);
  launch_dot_partial<T, T>(x, x, n, part, nullptr, h->s);
  launch_finalize(FIN_POWER0, part, nullptr, h->lp + l, h->opt.cheb_degree, nullptr, h->s);
  // step: d = Dinv K x / ||previous d|| with x the previous d, unscaled (the 1 / ||d|| of the previous step is
  // applied after the product, so no scaling pass), and the power step in the norm kernel's last block
  for (int it = 0; it < 12; ++it) {
    h->apply<T>(l, it == 0 ? x : d, t, nullptr);
    launch_bj_apply_norm<T>(FebHandle::dinv<T>(V), t, d, V.ntotal, part, h->s, it == 0 ? nullptr : h->lp + l,
                            h->lp + l, pctr, h->opt.cheb_degree);
  }
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

// The levels' power iterations touch disjoint buffers (each level's vectors, stencil, term dots and its own
// reduction scratch), so level k runs on side stream k (power_fork); the handle's stream meanwhile builds the
// dense coarsest level, which reads none of them, and then joins the side streams (power_join): the set-up
// waits for the slowest of these chains instead of their sum.  No allocation is made on a side stream.
template <typename T>
int power_fork(FebHandle* h, double** part) {
  FebHandle& H = *h;
  const int nl = H.coarsest;
  *part = nullptr;
  if (nl <= 0) return FEB_OK;
  // kRedBlocks partial sums per level, then one arrival counter per level (zeroed; re-armed by its last block)
  FEB_TRY(H.pool.alloc(part, (size_t)kRedBlocks * nl + nl));
  unsigned int* ctrs = reinterpret_cast<unsigned int*>(*part + (size_t)kRedBlocks * nl);
  FEB_CUDA(cudaMemsetAsync(ctrs, 0, (size_t)nl * sizeof(double), H.s));
  FEB_CUDA(cudaEventRecord(H.ev_sync, H.s));
  cudaStream_t main = H.s;
  int st = FEB_OK;
  for (int k = 0; k < nl && st == FEB_OK; ++k) {
    if (!H.aux[k]) {
      H.aux[k] = g_streams.stream();
      H.aux_ev[k] = g_streams.event();   // timed: the set-up's span ends at the slowest chain
      if (!H.aux[k] || !H.aux_ev[k]) { set_last_error("side stream / event creation failed"); return FEB_ERR_CUDA; }
    }
    FEB_CUDA(cudaStreamWaitEvent(H.aux[k], H.ev_sync, 0));
    H.s = H.aux[k];
    st = power_iteration<T>(h, k, *part + (size_t)kRedBlocks * k, ctrs + 2 * k);
    H.s = main;
    FEB_CUDA(cudaEventRecord(H.aux_ev[k], H.aux[k]));
  }
  return st;
}

int power_join(FebHandle* h, double* part) {
  FebHandle& H = *h;
  for (int k = 0; k < H.coarsest; ++k) FEB_CUDA(cudaStreamWaitEvent(H.s, H.aux_ev[k], 0));
  H.pool.free(part);
  return FEB_OK;
}

// ------------------------------------------------------------------------------------------------ autotuner
// Launch shape of the fine K.u (warps per CTA x node planes per CTA), picked by timing every candidate
// on this operator and cached per (grid, material model, split copies) for the process lifetime.
struct TuneKey {
  int nx, ny, nz, mode, copies, tc, pair;
  bool operator<(const TuneKey& o) const {
    return std::tie(nx, ny, nz, mode, copies, tc, pair) < std::tie(o.nx, o.ny, o.nz, o.mode, o.copies, o.tc, o.pair);
  }
};
struct Tuned {
  KuConfig k32, k64;
  PairConfig p32, p64;
};
std::mutex g_tune_mu;
std::map<TuneKey, Tuned> g_tune_cache;

// FEB_KU_TC: "0" keeps the FP32 K.u off the tensor cores, "1" puts it there without tuning (tests, profiling)
int env_tc() {
  const char* e = std::getenv("FEB_KU_TC");
  return (e && *e) ? (e[0] == '1' ? 1 : 0) : -1;
}

// average time of 3 products after 2 warm-up products (ms)
template <typename T>
int time_apply(FebHandle* h, T* u, T* y, float* ms) {
  for (int w = 0; w < 2; ++w) h->apply<T>(0, u, y, nullptr);
  FEB_TRY(h->tune_events());
  FEB_CUDA(cudaEventRecord(h->tev0, h->s));
  for (int r = 0; r < 3; ++r) h->apply<T>(0, u, y, nullptr);
  FEB_CUDA(cudaEventRecord(h->tev1, h->s));
  FEB_CUDA(cudaEventSynchronize(h->tev1));
  FEB_CUDA(cudaEventElapsedTime(ms, h->tev0, h->tev1));
  return FEB_OK;
}

template <typename T>
int tune_one(FebHandle* h, KuConfig* best, T* u, T* y) {
  std::vector<KuConfig> cand;
  const bool tc = std::is_same<T, float>::value && h->tc_ok;
  if (tc && env_tc() == 1) {
    *best = KuConfig{16, 16, 1};
    return FEB_OK;
  }
  for (int ty : {8, 12, 16})
    for (int zc : {6, 8, 12, 16, 24, 32}) cand.push_back(KuConfig{ty, zc, 0});
  if (tc)
    for (int zc : {8, 12, 16, 24, 32}) cand.push_back(KuConfig{16, zc, 1});
  float best_ms = 1e30f;
  for (const KuConfig& c : cand) {
    KuConfig& slot = std::is_same<T, double>::value ? h->ku64 : h->ku32;
    slot = c;
    float ms = 0.f;
    FEB_TRY(time_apply<T>(h, u, y, &ms));
    if (ms < best_ms) { best_ms = ms; *best = c; }
  }
  return FEB_OK;
}

// z chunks that fill 1 to 4 whole waves of resident CTAs, plus a few fixed sizes
template <typename T>
std::vector<int> wave_chunks(FebHandle* h, int wy, bool smooth) {
  int sms = kSmCount, dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int per_sm = fine_pair_blocks_per_sm<T>(h->mode, h->P32.cube, wy, smooth);
  const int txy = fine_pair_tiles_xy(h->nx + 1, h->ny + 1, wy);
  const int nzn = h->nz + 1;
  std::vector<int> zcs = {8, 16, 32};
  for (int waves = 1; waves <= 4; ++waves) {
    const int nbz = std::max(1, (waves * sms * per_sm) / std::max(txy, 1));
    zcs.push_back(std::max(2, div_up(nzn, nbz)));
  }
  std::sort(zcs.begin(), zcs.end());
  zcs.erase(std::unique(zcs.begin(), zcs.end()), zcs.end());
  return zcs;
}

// launch shapes of the paired kernel: products (warps per CTA x node planes per CTA) and smoothing steps
// (node planes per CTA at 8 warps), each timed on this operator
template <typename T>
int tune_pair(FebHandle* h, PairConfig* best, T* u, T* y, T* y2, T* y3) {
  PairConfig& slot = std::is_same<T, double>::value ? h->pc64 : h->pc32;
  const bool wide = std::is_same<T, float>::value && h->P32.cube;
  float best_ms = 1e30f;
  for (int wy : {8, 16}) {
    if (wy == 16 && !wide) continue;
    for (int zc : wave_chunks<T>(h, wy, false)) {
      slot.wy = wy;
      slot.zchunk = zc;
      float ms = 0.f;
      FEB_TRY(time_apply<T>(h, u, y, &ms));
      if (ms < best_ms) { best_ms = ms; best->wy = wy; best->zchunk = zc; }
    }
  }
  slot.wy = best->wy;
  slot.zchunk = best->zchunk;
  SmoothArgs<T> A;
  A.r_in = u; A.r_out = y; A.x_in = u; A.x_out = y2; A.d_out = y3;   // no parameters: a1 = a2 = 0, same traffic
  best_ms = 1e30f;
  for (int zc : wave_chunks<T>(h, 8, true)) {
    slot.zchunk_smooth = zc;
    for (int w = 0; w < 2; ++w) h->pair_run<T>(u, nullptr, &A, nullptr);
    FEB_TRY(h->tune_events());
    FEB_CUDA(cudaEventRecord(h->tev0, h->s));
    for (int r = 0; r < 3; ++r) h->pair_run<T>(u, nullptr, &A, nullptr);
    FEB_CUDA(cudaEventRecord(h->tev1, h->s));
    FEB_CUDA(cudaEventSynchronize(h->tev1));
    float ms = 0.f;
    FEB_CUDA(cudaEventElapsedTime(&ms, h->tev0, h->tev1));
    if (ms < best_ms) { best_ms = ms; best->zchunk_smooth = zc; }
  }
  slot = *best;
  return FEB_OK;
}

int autotune_ku(FebHandle* h) {
  TuneKey key{h->nx, h->ny, h->nz, h->mode, h->ntotal > h->nnode ? 1 : 0, h->tc_ok ? 2 + env_tc() : 0,
              h->pair_ok ? (h->P32.cube ? 2 : 1) : 0};
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      h->ku32 = it->second.k32;
      h->ku64 = it->second.k64;
      h->pc32 = it->second.p32;
      h->pc64 = it->second.p64;
      return FEB_OK;
    }
  }
  const char* env = std::getenv("FEB_KU_CONFIG");     // "ty,zchunk" pins the per-cell kernel's shape
  const char* penv = std::getenv("FEB_PAIR_CONFIG");  // "wy,zchunk" pins the paired kernel's shape
  bool pinned = false, ppinned = false;
  if (env && *env) {
    int ty = 16, zc = 16;
    if (std::sscanf(env, "%d,%d", &ty, &zc) == 2) {
      h->ku32 = h->ku64 = KuConfig{ty, zc, 0};
      pinned = true;
    }
  }
  if (h->tc_ok && env_tc() == 1) h->ku32 = KuConfig{16, 16, 1};
  if (penv && *penv) {      // "wy,zchunk[,zchunk_smooth]"
    int wy = 8, zc = 16, zs = 0;
    const int got = std::sscanf(penv, "%d,%d,%d", &wy, &zc, &zs);
    if (got >= 2) {
      if (got < 3) zs = zc;
      h->pc32 = PairConfig{(wy == 16 && h->P32.cube) ? 16 : 8, zc, zs};
      h->pc64 = PairConfig{8, zc, zs};
      ppinned = true;
    }
  }
  const bool need_cell = !h->pair_ok && !pinned, need_pair = h->pair_ok && !ppinned;
  if (!need_cell && !need_pair) return FEB_OK;
  const size_t n = 3 * (size_t)h->ntotal;
  double *u64 = nullptr, *y64 = nullptr, *y2 = nullptr, *y3 = nullptr;
  FEB_TRY(h->pool.zeros(&u64, n));
  FEB_TRY(h->pool.alloc(&y64, n));
  if (need_pair) {
    FEB_TRY(h->pool.alloc(&y2, n));
    FEB_TRY(h->pool.alloc(&y3, n));
  }
  Tuned t{h->ku32, h->ku64, h->pc32, h->pc64};
  if (need_cell) {
    FEB_TRY(tune_one<float>(h, &t.k32, (float*)u64, (float*)y64));
    FEB_TRY(tune_one<double>(h, &t.k64, u64, y64));
  }
  if (need_pair) {
    FEB_TRY(tune_pair<float>(h, &t.p32, (float*)u64, (float*)y64, (float*)y2, (float*)y3));
    FEB_TRY(tune_pair<double>(h, &t.p64, u64, y64, y2, y3));
  }
  h->pool.free(u64);
  h->pool.free(y64);
  h->pool.free(y2);
  h->pool.free(y3);
  h->ku32 = t.k32;
  h->ku64 = t.k64;
  h->pc32 = t.p32;
  h->pc64 = t.p64;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune_cache[key] = t;
  return FEB_OK;
}

// Tensor-core operand of the FP32 level-0 K.u: on equal cubic cells of edge h the ISO element matrices are
// h K(1) with 72 K_mu(1), 72 K_lambda(1) integer and the one-point 16 K_lambda(1) = s s^T, s[3l+c] = +-1 by
// bit c of l.  Read off the device element operator for the unit cube, checked to be those integers, laid
// out as the kernel's B table: [face cz][node row b][output n][4a + c] in BF16 (exact).  Leaves tc_ok false
// for other grids or models.
// Paired-row level-0 operator (fine_pair.cu): material ids of the regular cells (FEB_KU_PAIR=0 keeps the
// per-cell kernels), flags of the grid nodes that receive sparse contributions, the cell-pair words, the
// sparse accumulators and the symmetric level-0 block-Jacobi inverse.  Leaves pair_ok false when more than
// kMaxMatIds - 1 distinct materials occur (or on a hash collision).
template <int W>
int setup_pair(FebHandle* h, const double* mat_s64) {
  FebHandle& H = *h;
  const char* env = std::getenv("FEB_KU_PAIR");
  if (env && env[0] == '0') return FEB_OK;
  const int64_t ncell = (int64_t)H.nx * H.ny * H.nz;
  const int nxn = H.nx + 1, nyn = H.ny + 1, nzn = H.nz + 1;
  const int mp = nyn / 2 + 1;
  unsigned long long* keys = nullptr;
  double* vals = nullptr;
  uint8_t *ids = nullptr, *flag = nullptr;
  int* status = nullptr;
  uint16_t* cellpair = nullptr;
  FEB_TRY(H.pool.zeros(&keys, kMaxMatIds));
  FEB_TRY(H.pool.zeros(&vals, (size_t)W * kMaxMatIds));
  FEB_TRY(H.pool.alloc(&ids, ncell));
  FEB_TRY(H.pool.zeros(&flag, H.nnode));
  FEB_TRY(H.pool.zeros(&status, 1));
  FEB_TRY(H.pool.alloc(&cellpair, (size_t)nxn * mp * nzn));
  launch_mat_ids<W>(mat_s64, ncell, keys, vals, ids, status, H.s);
  launch_flag_nodes(H.F64.pen_node, H.F64.npen, H.F64.irr_nodes, H.F64.nirr, H.F64.row_dof, H.F64.nrow, H.nnode, flag,
                    H.s);
  launch_pack_pairs<W>(H.nx, H.ny, H.nz, mp, ids, flag, mat_s64, vals, cellpair, status, H.s);
  FEB_CUDA(cudaGetLastError());
  int st = 0;
  FEB_CUDA(cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, H.s));
  FEB_CUDA(cudaStreamSynchronize(H.s));
  H.pool.free(ids);
  H.pool.free(flag);
  H.pool.free(keys);
  H.pool.free(status);
  if (st != 0) {
    H.pool.free(cellpair);
    H.pool.free(vals);
    return FEB_OK;
  }
  const size_t n3 = 3 * (size_t)H.ntotal;
  float* tsp32 = nullptr;
  double* tsp64 = nullptr;
  FEB_TRY(H.pool.zeros(&tsp32, n3));
  FEB_TRY(H.pool.zeros(&tsp64, n3));
  FEB_TRY(H.pool.alloc(&H.D6_32, 6 * (size_t)H.ntotal));
  FEB_TRY(H.pool.alloc(&H.D6_64, 6 * (size_t)H.ntotal));
  launch_dinv6<float>(H.L[0].Dinv64, H.ntotal, H.D6_32, H.s);
  launch_dinv6<double>(H.L[0].Dinv64, H.ntotal, H.D6_64, H.s);
  FEB_CUDA(cudaGetLastError());
  const double hc = H.xe[1] - H.xe[0];
  auto uniform = [&](const std::vector<double>& e) {
    for (size_t i = 0; i + 1 < e.size(); ++i)
      if (std::fabs((e[i + 1] - e[i]) - hc) > 1e-12 * hc) return false;
    return true;
  };
  const bool cube = H.mode == MAT_ISO_SRI && hc > 0.0 && uniform(H.xe) && uniform(H.ye) && uniform(H.ze);
  auto fill = [&](auto& P, const auto& F, auto* tsp, const auto* d6) {
    P.nx = H.nx; P.ny = H.ny; P.nz = H.nz; P.nxn = nxn; P.nyn = nyn; P.nzn = nzn; P.mp = mp;
    P.nnode = H.nnode; P.ntotal = H.ntotal;
    P.cellpair = cellpair; P.mtab = vals; P.nmat = kMaxMatIds;
    P.cube = cube; P.h = hc;
    P.dx = F.dx; P.dy = F.dy; P.dz = F.dz; P.idx = F.idx; P.idy = F.idy; P.idz = F.idz;
    P.tsp = tsp; P.dinv6 = d6;
  };
  fill(H.P32, H.F32, tsp32, H.D6_32);
  fill(H.P64, H.F64, tsp64, H.D6_64);
  FEB_TRY(prepare_fine_pair(H.mode, cube));
  H.pc32 = PairConfig{cube ? 16 : 8, 16};
  H.pc64 = PairConfig{8, 16};
  H.pair_ok = true;
  return FEB_OK;
}

int setup_tc(FebHandle* h) {
  FebHandle& H = *h;
  if ((H.mode != MAT_ISO_SRI && H.mode != MAT_ISO_FULL) || env_tc() == 0) return FEB_OK;
  const double hc = H.xe[1] - H.xe[0];
  auto uniform = [&](const std::vector<double>& e) {
    for (size_t i = 0; i + 1 < e.size(); ++i)
      if (std::fabs((e[i + 1] - e[i]) - hc) > 1e-12 * hc) return false;
    return true;
  };
  if (!(hc > 0.0) || !uniform(H.xe) || !uniform(H.ye) || !uniform(H.ze)) return FEB_OK;
  const bool sri = H.mode == MAT_ISO_SRI;
  double* d = nullptr;
  FEB_TRY(H.pool.alloc(&d, 1152));
  if (sri) launch_unit_element<MAT_ISO_SRI>(d, H.s);
  else launch_unit_element<MAT_ISO_FULL>(d, H.s);
  std::vector<double> K(1152);
  FEB_CUDA(cudaMemcpyAsync(K.data(), d, 1152 * sizeof(double), cudaMemcpyDeviceToHost, H.s));
  FEB_CUDA(cudaStreamSynchronize(H.s));
  H.pool.free(d);
  const double* KL = K.data();
  const double* KM = K.data() + 576;
  int IM[24][24], IL[24][24], sg[24];
  for (int r = 0; r < 24; ++r) sg[r] = (((r / 3) >> (r % 3)) & 1) ? 1 : -1;
  for (int r = 0; r < 24; ++r)
    for (int c = 0; c < 24; ++c) {
      const double vm = 72.0 * KM[r * 24 + c], vl = 72.0 * KL[r * 24 + c];
      IM[r][c] = (int)std::lround(vm);
      IL[r][c] = (int)std::lround(vl);
      if (std::fabs(vm - IM[r][c]) > 1e-9 || std::abs(IM[r][c]) > 256) return FEB_OK;
      if (sri ? std::fabs(16.0 * KL[r * 24 + c] - sg[r] * sg[c]) > 1e-9
              : (std::fabs(vl - IL[r][c]) > 1e-9 || std::abs(IL[r][c]) > 256))
        return FEB_OK;
    }
  const int N = sri ? tc_columns<MAT_ISO_SRI>() : tc_columns<MAT_ISO_FULL>();
  std::vector<uint16_t> tab((size_t)4 * N * 8, 0);
  for (int cz = 0; cz < 2; ++cz)
    for (int b = 0; b < 2; ++b)
      for (int n = 0; n < N; ++n)
        for (int a = 0; a < 2; ++a)
          for (int c = 0; c < 3; ++c) {
            const int kd = 3 * (a + 2 * b + 4 * cz) + c;
            int v = 0;
            if (n < 24) v = IM[n][kd];
            else if (sri) v = (n == 24) ? sg[kd] : 0;
            else v = IL[n - 24][kd];
            const float fv = (float)v;
            uint32_t bits;
            std::memcpy(&bits, &fv, 4);
            tab[((size_t)(cz * 2 + b) * N + n) * 8 + 4 * a + c] = (uint16_t)(bits >> 16);   // exact: |v| <= 256
          }
  uint16_t* dtab = nullptr;
  FEB_TRY(H.pool.upload(&dtab, tab.data(), tab.size()));
  FEB_TRY(H.pool.zeros(&H.tc_status, 1));
  FEB_CUDA(sri ? prepare_fine_tc<MAT_ISO_SRI>() : prepare_fine_tc<MAT_ISO_FULL>());
  H.F32.tc_b = dtab;
  H.F32.tc_hmu = (float)(hc / 72.0);
  H.F32.tc_hlam = (float)(sri ? hc / 16.0 : hc / 72.0);
  H.F32.tc_status = H.tc_status;
  H.tc_ok = true;
  return FEB_OK;
}

// the level-1 stencil can be summed directly from the fine cells: uniform widths per axis, even cell counts,
// isotropic model (FEB_GALERKIN_DIRECT=0 keeps the coarse-cell matrices)
bool galerkin_direct_ok(const FebHandle& H) {
  auto uniform = [](const std::vector<double>& e) {
    const double w0 = e[1] - e[0];
    for (size_t i = 0; i + 1 < e.size(); ++i)
      if (std::fabs((e[i + 1] - e[i]) - w0) > 1e-12 * std::fabs(w0)) return false;
    return w0 > 0.0;
  };
  const char* genv = std::getenv("FEB_GALERKIN_DIRECT");
  return !(genv && genv[0] == '0') && H.mode != MAT_ORTHO && uniform(H.xe) && uniform(H.ye) && uniform(H.ze) &&
         H.nx % 2 == 0 && H.ny % 2 == 0 && H.nz % 2 == 0;
}

// Starts the level-1 stencil of a grid that will surely be coarsened on a side stream (the last one of the
// handle's side streams), right after the cells are prepared; build_hierarchy joins it.
template <int MODE>
int launch_level1_early(FebHandle& H) {
  const int cx = H.nx / 2 + 1, cy = H.ny / 2 + 1, cz = H.nz / 2 + 1;
  const int64_t n1 = (int64_t)cx * cy * cz;
  FEB_TRY(H.pool.zeros(&H.A1_early, 243 * (size_t)n1));
  FEB_TRY(H.pool.alloc(&H.A1_basis, 16 * 576));
  const int k = FebHandle::kAux - 1;
  if (!H.aux[k]) {
    H.aux[k] = g_streams.stream();
    H.aux_ev[k] = g_streams.event();   // timed: the set-up's span ends at the slowest chain
    if (!H.aux[k] || !H.aux_ev[k]) { set_last_error("side stream / event creation failed"); return FEB_ERR_CUDA; }
  }
  if (!H.A1_ev && !(H.A1_ev = g_streams.event())) { set_last_error("cudaEventCreate"); return FEB_ERR_CUDA; }
  FEB_CUDA(cudaEventRecord(H.ev_sync, H.s));
  FEB_CUDA(cudaStreamWaitEvent(H.aux[k], H.ev_sync, 0));
  const double a = H.xe[1] - H.xe[0], b = H.ye[1] - H.ye[0], c = H.ze[1] - H.ze[0];
  FEB_TRY(launch_galerkin_direct<MODE>(H.mat_all, H.nx, H.ny, a, b, c, H.A1_basis, H.A1_early, cx, cy, cz, H.aux[k]));
  FEB_CUDA(cudaEventRecord(H.A1_ev, H.aux[k]));
  return FEB_OK;
}

// The host pipeline of the extra entries (bounds check, merge, local / non-local classification, rank-1
// factoring) runs on a worker thread beside the cells stage and the early level-1 stencil.  The
// classification needs the split copies' grid positions, which the cells stage reads back: the worker waits
// for ready() (or gives up when the set-up fails first).  The used-node filter is applied by the caller
// afterwards, on the merged entries; dropping entries commutes with merging, so only when an entry is
// actually dropped are the classification and the factoring redone.
class ExtraPrep {
 public:
  Entries ex;                    // merged, every entry in range
  std::vector<char> is_local;    // both nodes within one cell of each other
  std::vector<char> taken;       // entries represented by `terms`
  Terms terms;
  char err[160] = {};            // bounds error (empty: none)
  int err_code = FEB_ERR_ARG;    // FEB_ERR_NOMEM when the worker ran out of host memory

  void start(const FebOperator* op, int64_t nnode, int64_t ntotal, int gx, int gy,
             const std::vector<int64_t>* orig_copy) {
    std::shared_future<void> go = ready_.get_future().share();
    th_ = std::thread([this, op, nnode, ntotal, gx, gy, orig_copy, go]() {
      try {
        run(op, nnode, ntotal, gx, gy, orig_copy, go);
      } catch (const std::exception& e) {   // nothing may escape a thread: report it as the set-up's error
        snprintf(err, sizeof(err), "extra entries: %s", e.what());
        err_code = FEB_ERR_NOMEM;
      }
    });
  }
  void run(const FebOperator* op, int64_t nnode, int64_t ntotal, int gx, int gy,
           const std::vector<int64_t>* orig_copy, const std::shared_future<void>& go) {
    ex.r.reserve(op->nextra); ex.c.reserve(op->nextra); ex.v.reserve(op->nextra);
    for (int64_t e2 = 0; e2 < op->nextra; ++e2) {
      const int64_t rr = op->extra_row[e2], cc = op->extra_col[e2];
      if (rr < 0 || cc < 0 || rr >= 3 * ntotal || cc >= 3 * ntotal) {
        snprintf(err, sizeof(err), "extra entry (%lld, %lld) out of range", (long long)rr, (long long)cc);
        return;
      }
      ex.r.push_back(rr); ex.c.push_back(cc); ex.v.push_back(op->extra_val[e2]);
    }
    coo_merge(ex);
    go.wait();
    if (!ok_.load(std::memory_order_acquire)) return;
    classify(nnode, gx, gy, *orig_copy);
    taken = factor_nonlocal(ex, is_local, terms);
  }
  // the split copies' positions are in place (called once, on success)
  void ready() {
    ok_.store(true, std::memory_order_release);
    release();
  }
  void join() {
    release();
    if (th_.joinable()) th_.join();
  }
  ~ExtraPrep() { join(); }

  // grid coordinates by 32-bit unsigned division (grid node ids are below 2^31): two divisions per node
  void classify(int64_t nnode, int gx, int gy, const std::vector<int64_t>& orig_copy) {
    const uint32_t ugx = (uint32_t)gx, ugy = (uint32_t)gy;
    auto coords = [&](int64_t node, int& x, int& y, int& z) {
      const uint32_t a = (uint32_t)(node < nnode ? node : orig_copy[node - nnode]), q = a / ugx;
      x = int(a - q * ugx); z = int(q / ugy); y = int(q - (uint32_t)z * ugy);
    };
    is_local.assign(ex.size(), 0);
    auto slice = [&](size_t lo, size_t hi) {
      for (size_t e2 = lo; e2 < hi; ++e2) {
        int ax, ay, az, bx, by, bz;
        coords(ex.r[e2] / 3, ax, ay, az);
        coords(ex.c[e2] / 3, bx, by, bz);
        is_local[e2] = std::abs(ax - bx) <= 1 && std::abs(ay - by) <= 1 && std::abs(az - bz) <= 1;
      }
    };
    const size_t n = ex.size();
    if (n >= 32768 && std::thread::hardware_concurrency() >= 4) {   // independent entries: 4 slices
      std::vector<std::thread> th;
      for (int p = 1; p < 4; ++p) th.emplace_back(slice, n * p / 4, n * (p + 1) / 4);
      slice(0, n / 4);
      for (auto& t : th) t.join();
    } else {
      slice(0, n);
    }
  }

 private:
  void release() {
    if (!released_) { released_ = true; ready_.set_value(); }
  }
  std::promise<void> ready_;
  std::atomic<bool> ok_{false};
  bool released_ = false;
  std::thread th_;
};

template <int W>
int setup_level0(FebHandle* h, const FebOperator* op) {
  FebHandle& H = *h;
  cudaStream_t s = H.s;
  const int64_t ncell = (int64_t)H.nx * H.ny * H.nz;
  Level& V = H.L[0];
  V.nx = H.nx + 1; V.ny = H.ny + 1; V.nz = H.nz + 1;
  V.nnode = H.nnode; V.ntotal = H.ntotal;
  V.coord[0] = H.xe; V.coord[1] = H.ye; V.coord[2] = H.ze;
  ExtraPrep xp;
  if (op->nextra > 0) xp.start(op, H.nnode, H.ntotal, H.nx + 1, H.ny + 1, &H.orig_copy_h);
  // per-axis widths
  std::vector<double> w64[3], iw64[3];
  std::vector<float> w32[3], iw32[3];
  const std::vector<double>* e[3] = {&H.xe, &H.ye, &H.ze};
  double* dw64[3]; double* diw64[3]; float* dw32[3]; float* diw32[3];
  for (int d = 0; d < 3; ++d) {
    for (size_t i = 0; i + 1 < e[d]->size(); ++i) {
      double w = (*e[d])[i + 1] - (*e[d])[i];
      w64[d].push_back(w); iw64[d].push_back(1.0 / w);
      w32[d].push_back((float)w); iw32[d].push_back((float)(1.0 / w));
    }
    FEB_TRY(H.pool.upload(&dw64[d], w64[d].data(), w64[d].size()));
    FEB_TRY(H.pool.upload(&diw64[d], iw64[d].data(), iw64[d].size()));
    FEB_TRY(H.pool.upload(&dw32[d], w32[d].data(), w32[d].size()));
    FEB_TRY(H.pool.upload(&diw32[d], iw32[d].data(), iw32[d].size()));
  }
  FEB_TRY(H.pool.upload(&H.xe_d, H.xe.data(), H.xe.size()));
  FEB_TRY(H.pool.upload(&H.ye_d, H.ye.data(), H.ye.size()));
  FEB_TRY(H.pool.upload(&H.ze_d, H.ze.data(), H.ze.size()));
  // cells
  double *mat_s64;
  float* mat_s32;
  uint8_t* irr_flag;
  FEB_TRY(H.pool.alloc(&H.mat_all, W * ncell));
  FEB_TRY(H.pool.alloc(&mat_s64, W * ncell));
  FEB_TRY(H.pool.alloc(&mat_s32, W * ncell));
  FEB_TRY(H.pool.alloc(&irr_flag, ncell));
  FEB_TRY(H.pool.zeros(&V.used, H.ntotal));
  k_prepare_cells<W><<<div_up(ncell, kThreads), kThreads, 0, s>>>(H.nx, H.ny, H.nz, op->mat, H.mode, op->active, op->cn,
                                                                  H.mat_all, mat_s64, mat_s32, irr_flag, V.used); note_launch();
  FEB_CUDA(cudaGetLastError());
  // irregular cells, in ascending cell-id order
  int nirr = 0;
  int *irr_cell = nullptr, *irr_nodes = nullptr;
  double* irr_m64 = nullptr;
  float* irr_m32 = nullptr;
  if (op->cn) {
    int64_t* sel = nullptr;
    int* nsel = nullptr;
    FEB_TRY(H.pool.alloc(&sel, ncell));
    FEB_TRY(H.pool.alloc(&nsel, 1));
    size_t tb = 0;
    thrust::counting_iterator<int64_t> cnt(0);
    FEB_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, cnt, irr_flag, sel, nsel, ncell, s));
    uint8_t* tmp = nullptr;
    FEB_TRY(H.pool.alloc(&tmp, tb));
    FEB_CUDA(cub::DeviceSelect::Flagged(tmp, tb, cnt, irr_flag, sel, nsel, ncell, s));
    FEB_CUDA(cudaMemcpyAsync(&nirr, nsel, sizeof(int), cudaMemcpyDeviceToHost, s));
    FEB_CUDA(cudaStreamSynchronize(s));
    if (nirr > 0) {
      FEB_TRY(H.pool.alloc(&irr_cell, nirr));
      FEB_TRY(H.pool.alloc(&irr_nodes, 8 * (size_t)nirr));
      FEB_TRY(H.pool.alloc(&irr_m64, W * (size_t)nirr));
      FEB_TRY(H.pool.alloc(&irr_m32, W * (size_t)nirr));
      k_build_irregular<W><<<div_up(nirr, kThreads), kThreads, 0, s>>>(H.nx, H.ny, H.nz, sel, nirr, op->mat, H.mode,
                                                                        op->cn, irr_cell, irr_nodes, irr_m64, irr_m32); note_launch();
      FEB_CUDA(cudaGetLastError());
    }
    H.pool.free(tmp); H.pool.free(sel); H.pool.free(nsel);
  }
  H.pool.free(irr_flag);
  // copies
  if (H.ntotal > H.nnode) {
    if (!op->orig) { set_last_error("feb_create: nnode_total > grid nodes needs orig"); return FEB_ERR_ARG; }
    FEB_TRY(H.pool.alloc(&H.orig_copy, H.ntotal - H.nnode));
    k_orig_copy<<<div_up(H.ntotal - H.nnode, kThreads), kThreads, 0, s>>>(op->orig, H.nnode, H.ntotal, H.orig_copy); note_launch();
    std::vector<int> oc(H.ntotal - H.nnode);
    FEB_CUDA(cudaMemcpyAsync(oc.data(), H.orig_copy, oc.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    FEB_CUDA(cudaStreamSynchronize(s));
    H.orig_copy_h.assign(oc.begin(), oc.end());
  }
  xp.ready();
  // a grid far above the coarsest size always gets level 1: its stencil starts now, beside the host work below
  if (H.opt.max_levels >= 2 && 3 * H.nnode > 8 * (int64_t)H.opt.min_dofs && galerkin_direct_ok(H)) {
    if (H.mode == MAT_ISO_SRI) FEB_TRY(launch_level1_early<MAT_ISO_SRI>(H));
    else FEB_TRY(launch_level1_early<MAT_ISO_FULL>(H));
  }
  H.stage_mark();   // 1: cells, irregular list, copies
  g_prof.mark("L0 cells/irregular/copies", s);
  std::vector<uint8_t> used_h(H.ntotal);
  FEB_CUDA(cudaMemcpyAsync(used_h.data(), V.used, H.ntotal, cudaMemcpyDeviceToHost, s));
  FEB_CUDA(cudaStreamSynchronize(s));
  if (op->nmark > 0) {     // nodes of a matrix-only operator
    for (int64_t e2 = 0; e2 < op->nmark; ++e2) {
      int64_t node = op->mark_used[e2];
      if (node < 0 || node >= H.ntotal) { set_last_error("mark_used node %lld out of range", (long long)node); return FEB_ERR_ARG; }
      used_h[node] = 1;
    }
    FEB_CUDA(cudaMemcpyAsync(V.used, used_h.data(), H.ntotal, cudaMemcpyHostToDevice, s));
    FEB_CUDA(cudaStreamSynchronize(s));
  }
  g_prof.mark("L0 used mask to host", s);
  // penalties (entries on unused nodes are dropped, fe/solver.py:213-215)
  std::vector<int> pn;
  std::vector<double> pk;
  std::vector<float> pkf;
  pn.reserve(op->npen); pk.reserve(3 * op->npen); pkf.reserve(3 * op->npen);
  for (int64_t e2 = 0; e2 < op->npen; ++e2) {
    int64_t node = op->pen_node[e2];
    if (node < 0 || node >= H.ntotal) { set_last_error("penalty node %lld out of range", (long long)node); return FEB_ERR_ARG; }
    if (!used_h[node]) continue;
    pn.push_back((int)node);
    for (int c = 0; c < 3; ++c) { pk.push_back(op->pen_k[3 * e2 + c]); pkf.push_back((float)op->pen_k[3 * e2 + c]); }
  }
  H.npen = (int)pn.size();
  int* pen_node = nullptr;
  double* pen_k64 = nullptr;
  float* pen_k32 = nullptr;
  FEB_TRY(H.pool.upload(&pen_node, pn.data(), pn.size()));
  FEB_TRY(H.pool.upload(&pen_k64, pk.data(), pk.size()));
  FEB_TRY(H.pool.upload(&pen_k32, pkf.data(), pkf.size()));
  // extra matrix: all entries applied on level 0; local ones folded into the level-1 stencil on the
  // device, non-local ones projected through the levels on the host
  g_prof.mark("L0 penalties", s);
  xp.join();
  if (xp.err[0]) { set_last_error("%s", xp.err); return xp.err_code; }
  Entries& ex = xp.ex;
  std::vector<char>& is_local = xp.is_local;
  std::vector<char>& taken = xp.taken;
  V.terms = std::move(xp.terms);
  // entries on unused nodes are dropped (fe/solver.py:213-215); rare, and then the worker's classification
  // and factoring of the dropped set are redone on what remains
  size_t keep = 0;
  for (size_t e2 = 0; e2 < ex.size(); ++e2) keep += used_h[ex.r[e2] / 3] && used_h[ex.c[e2] / 3];
  if (keep < ex.size()) {
    Entries f;
    f.r.reserve(keep); f.c.reserve(keep); f.v.reserve(keep);
    for (size_t e2 = 0; e2 < ex.size(); ++e2)
      if (used_h[ex.r[e2] / 3] && used_h[ex.c[e2] / 3]) { f.r.push_back(ex.r[e2]); f.c.push_back(ex.c[e2]); f.v.push_back(ex.v[e2]); }
    ex = std::move(f);
    xp.classify(H.nnode, H.nx + 1, H.ny + 1, H.orig_copy_h);
    V.terms = Terms();
    taken = factor_nonlocal(ex, is_local, V.terms);
  }
  g_prof.mark("L0 extra entries (worker joined, used filter)", s);
  Csr c0;
  FEB_TRY(upload_csr(H.pool, ex, c0));
  g_prof.mark("L0 extra CSR upload", s);
  Entries loc;
  for (size_t e2 = 0; e2 < ex.size(); ++e2) {
    if (taken[e2]) continue;
    Entries& dst = is_local[e2] ? loc : V.nonlocal;
    dst.r.push_back(ex.r[e2]); dst.c.push_back(ex.c[e2]); dst.v.push_back(ex.v[e2]);
  }
  H.nlocal = (int)loc.size();
  if (H.nlocal) {
    std::vector<int> lr(loc.r.begin(), loc.r.end()), lc(loc.c.begin(), loc.c.end());
    FEB_TRY(H.pool.upload(&H.loc_r, lr.data(), lr.size()));
    FEB_TRY(H.pool.upload(&H.loc_c, lc.data(), lc.size()));
    FEB_TRY(H.pool.upload(&H.loc_v, loc.v.data(), loc.v.size()));
  }
  // device views
  FineView<double>& F = H.F64;
  FineView<float>& G = H.F32;
  F.nx = G.nx = H.nx; F.ny = G.ny = H.ny; F.nz = G.nz = H.nz;
  F.nxn = G.nxn = H.nx + 1; F.nyn = G.nyn = H.ny + 1; F.nzn = G.nzn = H.nz + 1;
  F.nnode = G.nnode = H.nnode; F.ntotal = G.ntotal = H.ntotal;
  F.dx = dw64[0]; F.dy = dw64[1]; F.dz = dw64[2]; F.idx = diw64[0]; F.idy = diw64[1]; F.idz = diw64[2];
  G.dx = dw32[0]; G.dy = dw32[1]; G.dz = dw32[2]; G.idx = diw32[0]; G.idy = diw32[1]; G.idz = diw32[2];
  F.mat = mat_s64; G.mat = mat_s32;
  F.nirr = G.nirr = nirr; F.irr_cell = G.irr_cell = irr_cell; F.irr_nodes = G.irr_nodes = irr_nodes;
  F.irr_mat = irr_m64; G.irr_mat = irr_m32;
  F.npen = G.npen = H.npen; F.pen_node = G.pen_node = pen_node; F.pen_k = pen_k64; G.pen_k = pen_k32;
  F.nrow = G.nrow = c0.nrow; F.row_dof = G.row_dof = c0.row_dof; F.row_ptr = G.row_ptr = c0.row_ptr;
  F.col = G.col = c0.col; F.val = c0.v64; G.val = c0.v32;
  // used nodes, diagonal blocks
  H.stage_mark();   // 2: penalties and extra entries (host sort / classification, uploads)
  FEB_TRY(count_mask(h, V.used, H.ntotal, &H.ndof));
  H.ndof *= 3;
  V.ndof = H.ndof;
  double* D = nullptr;
  FEB_TRY(H.pool.alloc(&D, 9 * (size_t)H.ntotal));
  switch (H.mode) {
    case MAT_ISO_SRI: launch_fine_diag<MAT_ISO_SRI>(F, D, s); break;
    case MAT_ISO_FULL: launch_fine_diag<MAT_ISO_FULL>(F, D, s); break;
    default: launch_fine_diag<MAT_ORTHO>(F, D, s); break;
  }
  FEB_TRY(H.pool.alloc(&V.Dinv64, 9 * (size_t)H.ntotal));
  FEB_TRY(H.pool.alloc(&V.Dinv32, 9 * (size_t)H.ntotal));
  launch_block_inverse(D, H.ntotal, V.Dinv64, V.Dinv32, s);
  FEB_CUDA(cudaGetLastError());
  H.pool.free(D);
  FEB_TRY(setup_pair<W>(h, mat_s64));
  H.stage_mark();   // 3: used nodes, level-0 diagonal blocks, paired-row operator
  g_prof.mark("L0 local upload, diag blocks, pair operator", s);
  // the autotuner's timings must not share the GPU with the early level-1 stencil: wait for it first (the
  // host work of stage 2 is longer than the stencil, so this wait is normally already satisfied)
  if (H.A1_early) FEB_CUDA(cudaStreamWaitEvent(s, H.A1_ev, 0));
  FEB_TRY(setup_tc(h));
  FEB_TRY(autotune_ku(h));
  H.stage_mark();   // 4: K.u autotuning (first handle of a grid shape only)
  g_prof.mark("L0 tensor-core operand, tuning", s);
  return FEB_OK;
}

int build_dense(FebHandle* h) {
  FebHandle& H = *h;
  Level& V = H.L[H.coarsest];
  const int64_t n = V.ntotal;
  std::vector<uint8_t> mask(n);
  FEB_CUDA(cudaMemcpyAsync(mask.data(), V.used, n, cudaMemcpyDeviceToHost, H.s));
  FEB_CUDA(cudaStreamSynchronize(H.s));
  std::vector<int> cmap(n, -1), klist;
  for (int64_t i = 0; i < n; ++i)
    if (mask[i]) { cmap[i] = (int)klist.size(); klist.push_back((int)i); }
  H.nd = 3 * (int)klist.size();
  if (H.nd == 0) { set_last_error("empty coarsest level"); return FEB_ERR_ARG; }
  // buffers are allocated (stream-ordered) on s; the assembly and the inverse run on dense_s from here, and
  // feb_create returns without waiting for them (FebHandle::settle joins them)
  FEB_TRY(H.pool.upload(&H.cmap, cmap.data(), cmap.size()));
  FEB_TRY(H.pool.upload(&H.klist, klist.data(), klist.size()));
  FEB_TRY(H.pool.zeros(&H.Minv, (size_t)H.nd * H.nd));
  int *dr = nullptr, *dc = nullptr;
  double* dv = nullptr;
  if (H.coarsest > 0 && V.sparse.size()) {
    std::vector<int> rr(V.sparse.r.begin(), V.sparse.r.end()), cc(V.sparse.c.begin(), V.sparse.c.end());
    FEB_TRY(H.pool.upload(&dr, rr.data(), rr.size()));
    FEB_TRY(H.pool.upload(&dc, cc.data(), cc.size()));
    FEB_TRY(H.pool.upload(&dv, V.sparse.v.data(), V.sparse.v.size()));
  }
  double* scratch = nullptr;
  FEB_TRY(H.pool.alloc(&scratch, dense_scratch_doubles(H.nd)));
  if (!H.dense_st) FEB_TRY(H.pool.zeros(&H.dense_st, 1));
  if (!H.dense_st_h && !(H.dense_st_h = g_pinned.take())) { set_last_error("cudaMallocHost"); return FEB_ERR_CUDA; }
  if (!H.dense_s) {
    H.dense_s = g_streams.stream();
    H.dense_ev = g_streams.event();
    if (!H.dense_s || !H.dense_ev) { set_last_error("side stream / event creation failed"); return FEB_ERR_CUDA; }
  }
  FEB_CUDA(cudaEventRecord(H.ev_sync, H.s));
  FEB_CUDA(cudaStreamWaitEvent(H.dense_s, H.ev_sync, 0));
  cudaStream_t ds = H.dense_s;
  if (H.coarsest == 0) {
    switch (H.mode) {
      case MAT_ISO_SRI: launch_dense_from_fine<MAT_ISO_SRI>(H.F64, H.cmap, H.Minv, H.nd, ds); break;
      case MAT_ISO_FULL: launch_dense_from_fine<MAT_ISO_FULL>(H.F64, H.cmap, H.Minv, H.nd, ds); break;
      default: launch_dense_from_fine<MAT_ORTHO>(H.F64, H.cmap, H.Minv, H.nd, ds); break;
    }
  } else {
    launch_dense_from_stencil(V.A64, V.nx, V.ny, V.nz, H.cmap, H.Minv, H.nd, ds);
    if (dr) launch_dense_add_entries((int)V.sparse.size(), dr, dc, dv, H.cmap, H.Minv, H.nd, ds);
    launch_dense_add_terms(V.nterms, V.t_ptr, V.t_dof, V.t_val64, V.t_lam64, H.cmap, H.Minv, H.nd, ds);
  }
  FEB_CUDA(cudaMemsetAsync(H.dense_st, 0, sizeof(int), ds));
  launch_dense_invert(H.Minv, H.nd, scratch, H.dense_st, ds);
  FEB_CUDA(cudaGetLastError());
  FEB_CUDA(cudaMemcpyAsync(H.dense_st_h, H.dense_st, sizeof(int), cudaMemcpyDeviceToHost, ds));
  FEB_CUDA(cudaEventRecord(H.dense_ev, ds));
  H.pending = true;
  for (void* p : {(void*)scratch, (void*)dr, (void*)dc, (void*)dv})
    if (p) H.deferred_free.push_back(p);
  return FEB_OK;
}

int build_hierarchy(FebHandle* h) {
  FebHandle& H = *h;
  const bool f32 = H.opt.precision != FEB_PREC_FP64;
  if (H.opt.max_levels <= 0) {   // operator only: K.u is available, no multigrid (feb_solve refuses)
    H.coarsest = -1;
    return FEB_OK;
  }
  const int maxl = std::min(H.opt.max_levels, kMaxLevels);
  int l = 0;
  while (true) {
    Level& V = H.L[l];
    if (V.ndof <= H.opt.min_dofs || l == maxl - 1) { H.coarsest = l; break; }
    // transfer l -> l+1
    for (int d = 0; d < 3; ++d) V.ax[d] = make_axis(V.coord[d]);
    FEB_TRY(upload_transfer(H.pool, V));
    if (l == 0) FEB_TRY(upload_copy_gather(H.pool, V, H.orig_copy_h));
    g_prof.mark("Lk transfer", H.s);
    H.L.emplace_back();
    Level& C = H.L.back();
    Level& F = H.L[l];   // reference again after emplace_back
    C.nx = F.ax[0].nc; C.ny = F.ax[1].nc; C.nz = F.ax[2].nc;
    C.nnode = C.ntotal = (int64_t)C.nx * C.ny * C.nz;
    for (int d = 0; d < 3; ++d) C.coord[d] = F.ax[d].coarse;
    FEB_TRY(H.pool.alloc(&C.used, C.ntotal));
    launch_kept_mask(F.P, F.used, C.used, H.s);
    int64_t kept = 0;
    FEB_TRY(count_mask(h, C.used, C.ntotal, &kept));
    C.ndof = 3 * kept;
    g_prof.mark("Lk kept mask + count", H.s);
    const bool early = l == 0 && H.A1_early && C.nx == H.nx / 2 + 1 && C.ny == H.ny / 2 + 1 && C.nz == H.nz / 2 + 1;
    if (early) {          // the stencil was started on a side stream during the level-0 set-up
      C.A64 = H.A1_early;
      H.A1_early = nullptr;
      FEB_CUDA(cudaStreamWaitEvent(H.s, H.A1_ev, 0));
    } else {
      FEB_TRY(H.pool.zeros(&C.A64, 243 * (size_t)C.ntotal));
    }
    if (l == 0) {
      // uniform widths per axis, even cell counts, isotropic model: the stencil is summed directly from the
      // fine cells' materials; otherwise coarse-cell matrices first, then the node stencil
      const bool direct = galerkin_direct_ok(H) && C.nx == H.nx / 2 + 1 && C.ny == H.ny / 2 + 1 &&
                          C.nz == H.nz / 2 + 1;
      if (direct) {
        double* basis = H.A1_basis;
        H.A1_basis = nullptr;
        if (!early) {
          if (!basis) FEB_TRY(H.pool.alloc(&basis, 16 * 576));
          const double a = H.xe[1] - H.xe[0], b = H.ye[1] - H.ye[0], c = H.ze[1] - H.ze[0];
          if (H.mode == MAT_ISO_SRI)
            FEB_TRY(launch_galerkin_direct<MAT_ISO_SRI>(H.mat_all, H.nx, H.ny, a, b, c, basis, C.A64, C.nx, C.ny, C.nz, H.s));
          else
            FEB_TRY(launch_galerkin_direct<MAT_ISO_FULL>(H.mat_all, H.nx, H.ny, a, b, c, basis, C.A64, C.nx, C.ny, C.nz, H.s));
        }
        // interior patterns of the compressed level-1 stencil (tags follow once the half stencil exists)
        const char* cenv = std::getenv("FEB_SYM_COMPRESS");   // opt-in: measured slower on the hindfoot
        if (H.pair_ok && cenv && cenv[0] == '1') {
          FEB_TRY(H.pool.alloc(&C.pat64, 252));
          launch_sym_pattern(basis, C.pat64, H.s);
        }
        FEB_CUDA(cudaGetLastError());
        H.pool.free(basis);
      } else {
        double* KeC = nullptr;
        FEB_TRY(H.pool.alloc(&KeC, 576 * (size_t)(C.nx - 1) * (C.ny - 1) * (C.nz - 1)));
        switch (H.mode) {
          case MAT_ISO_SRI: launch_galerkin_cells<MAT_ISO_SRI>(H.F64, H.mat_all, F.P, KeC, C.A64, C.nx, C.ny, C.nz, H.s); break;
          case MAT_ISO_FULL: launch_galerkin_cells<MAT_ISO_FULL>(H.F64, H.mat_all, F.P, KeC, C.A64, C.nx, C.ny, C.nz, H.s); break;
          default: launch_galerkin_cells<MAT_ORTHO>(H.F64, H.mat_all, F.P, KeC, C.A64, C.nx, C.ny, C.nz, H.s); break;
        }
        FEB_CUDA(cudaGetLastError());
        H.pool.free(KeC);
      }
      launch_galerkin_penalty(F.P, F.nx, F.ny, F.nnode, H.orig_copy, H.npen, H.F64.pen_node, H.F64.pen_k, C.A64, C.nx,
                              C.ny, C.nz, C.ntotal, H.s);
      launch_galerkin_local(F.P, F.nx, F.ny, F.nnode, H.orig_copy, H.nlocal, H.loc_r, H.loc_c, H.loc_v, C.A64, C.nx,
                            C.ny, C.nz, C.ntotal, H.s);
    } else {
      double *T1 = nullptr, *T2 = nullptr;    // x coarsened, then y; z lands in C.A64
      FEB_TRY(H.pool.alloc(&T1, 243 * (size_t)C.nx * F.ny * F.nz));
      FEB_TRY(H.pool.alloc(&T2, 243 * (size_t)C.nx * C.ny * F.nz));
      launch_galerkin_axis(F.P.ax[0], 0, F.A64, F.nx, F.ny, F.nz, T1, C.nx, F.ny, F.nz, H.s);
      launch_galerkin_axis(F.P.ax[1], 1, T1, C.nx, F.ny, F.nz, T2, C.nx, C.ny, F.nz, H.s);
      launch_galerkin_axis(F.P.ax[2], 2, T2, C.nx, C.ny, F.nz, C.A64, C.nx, C.ny, C.nz, H.s);
      H.pool.free(T1);
      H.pool.free(T2);
    }
    FEB_CUDA(cudaGetLastError());
    g_prof.mark("Lk Galerkin product", H.s);
    C.nonlocal = project(F.nonlocal, F.ax, H.orig_copy_h, F.nnode, F.nx, F.ny);
    C.terms = project_terms(F.terms, F.ax, H.orig_copy_h, F.nnode, F.nx, F.ny);
    C.sparse = C.nonlocal;
    FEB_TRY(upload_node_csr(H.pool, C.sparse, C.nnode, C));
    FEB_TRY(upload_terms(H.pool, C.terms, C.nnode, C));
    g_prof.mark("Lk sparse project + upload", H.s);
    FEB_TRY(H.pool.alloc(&C.S64, 126 * (size_t)sym_np(C.nx, C.ny, C.nz)));
    launch_stencil_to_sym<double>(C.A64, C.nx, C.ny, C.nz, C.S64, H.s);
    if (C.pat64) {   // compressed level-1 stencil: tags of the uniform nodes, patterns and material table in T
      FEB_TRY(H.pool.alloc(&C.tag, C.ntotal));
      launch_sym_tags(C.S64, C.nx, C.ny, C.nz, H.P32.cellpair, H.nx + 1, H.P32.mp, H.P32.mtab, C.pat64, C.tag, H.s);
      C.tmat64 = const_cast<double*>(H.P32.mtab);
      if (f32) {
        FEB_TRY(H.pool.alloc(&C.pat32, 252));
        FEB_TRY(H.pool.alloc(&C.tmat32, 2 * kMaxMatIds));
        launch_convert<double, float>(C.pat64, C.pat32, 252, nullptr, H.s);
        launch_convert<double, float>(C.tmat64, C.tmat32, 2 * kMaxMatIds, nullptr, H.s);
      }
      FEB_CUDA(cudaGetLastError());
    }
    // FP16 copy scaled by a power of two (the compile-time-slot product reads it), else an FP32 copy
    if (f32 && !(H.opt.level_kernel & 8) && (H.opt.level_kernel & 3) != 1 && !C.tag) {
      FEB_TRY(H.pool.alloc(&C.S16, 126 * (size_t)sym_np(C.nx, C.ny, C.nz)));
      FEB_TRY(H.pool.alloc(&C.hscale, 2));
      launch_sym_to_half(C.S64, C.nx, C.ny, C.nz, reinterpret_cast<unsigned*>(C.hscale + 1), C.hscale, C.S16, H.s);
    } else if (f32) {
      FEB_TRY(H.pool.alloc(&C.S32, 126 * (size_t)sym_np(C.nx, C.ny, C.nz)));
      launch_stencil_to_sym<float>(C.A64, C.nx, C.ny, C.nz, C.S32, H.s);
    }
    g_prof.mark("Lk half stencils", H.s);
    l += 1;
    bool last = (C.ndof <= H.opt.min_dofs) || (l == maxl - 1);
    if (!last) {
      double* D = nullptr;
      FEB_TRY(H.pool.alloc(&D, 9 * (size_t)C.ntotal));
      launch_stencil_diag(C.A64, C.ntotal, D, H.s);
      std::vector<int> dr, dc;
      std::vector<double> dv;
      for (size_t e = 0; e < C.sparse.size(); ++e)
        if (C.sparse.r[e] / 3 == C.sparse.c[e] / 3) {
          dr.push_back((int)C.sparse.r[e]); dc.push_back((int)C.sparse.c[e]); dv.push_back(C.sparse.v[e]);
        }
      for (size_t t = 0; t < C.terms.size(); ++t)      // lam v_n v_n^T: the terms' 3x3 diagonal blocks
        for (int64_t a = C.terms.ptr[t]; a < C.terms.ptr[t + 1]; ++a)
          for (int64_t b = C.terms.ptr[t]; b < C.terms.ptr[t + 1]; ++b)
            if (C.terms.dof[a] / 3 == C.terms.dof[b] / 3) {
              dr.push_back((int)C.terms.dof[a]); dc.push_back((int)C.terms.dof[b]);
              dv.push_back(C.terms.lam[t] * C.terms.val[a] * C.terms.val[b]);
            }
      if (!dr.empty()) {
        int *ddr, *ddc;
        double* ddv;
        FEB_TRY(H.pool.upload(&ddr, dr.data(), dr.size()));
        FEB_TRY(H.pool.upload(&ddc, dc.data(), dc.size()));
        FEB_TRY(H.pool.upload(&ddv, dv.data(), dv.size()));
        launch_add_diag_entries((int)dr.size(), ddr, ddc, ddv, D, H.s);
      }
      FEB_TRY(H.pool.alloc(&C.Dinv64, 9 * (size_t)C.ntotal));
      if (f32) FEB_TRY(H.pool.alloc(&C.Dinv32, 9 * (size_t)C.ntotal));
      launch_block_inverse(D, C.ntotal, C.Dinv64, C.Dinv32, H.s);
      FEB_CUDA(cudaGetLastError());
      H.pool.free(D);
      g_prof.mark("Lk block-Jacobi", H.s);
    }
  }
  H.stage_mark();   // 5: transfers, Galerkin products, coarse diagonal blocks
  // work vectors and smoother parameters
  for (int k = 0; k <= H.coarsest; ++k) {
    Level& V = H.L[k];
    FEB_TRY(level_vectors<double>(H.pool, V, true, f32));
  }
  g_prof.mark("level work vectors", H.s);
  // The power steps run in FP64 for every precision: on the 160 x 112 x 96 hindfoot the FP32 estimate cost the
  // mixed solve 5 iterations (78 against 73; FP64 V-cycle 72).  FEB_POWER_FP32=1 runs them in the V-cycle's
  // precision instead (as rb/gpusolve.py:84-97 does in its multigrid dtype).
  const bool pw32 = f32 && env_flag("FEB_POWER_FP32");
  double* part = nullptr;
  const int pst = pw32 ? power_fork<float>(h, &part) : power_fork<double>(h, &part);
  if (pst != FEB_OK) { power_join(h, part); return pst; }
  H.stage_mark();   // 6: work vectors, power iterations started on the side streams
  g_prof.mark("power iterations (launched)", H.s);
  // the dense coarsest level runs on its own stream beside the power iterations; neither is waited for
  // here: the caller's next steps overlap them, and settle() joins them (stage 6's time is measured there)
  const int dst = build_dense(h);
  if (dst != FEB_OK) { power_join(h, part); return dst; }
  H.pending = true;
  H.deferred_free.push_back(part);
  if (g_prof.on) {
    FEB_TRY(H.settle());
    g_prof.mark("dense coarsest inverse, power iterations (joined)", H.s);
  }
  // the full stencils only feed the Galerkin products and the dense level; the FP64 half stencils of an FP32
  // V-cycle only the power iterations: all are released once the deferred work is joined
  for (int k = 1; k <= H.coarsest; ++k) {
    H.deferred_free.push_back(H.L[k].A64);
    H.L[k].A64 = nullptr;
    if (f32 && !pw32) { H.deferred_free.push_back(H.L[k].S64); H.L[k].S64 = nullptr; }
  }
  if (!H.pending) {                              // joined above (set-up profiling)
    for (void* p : H.deferred_free) H.pool.free(p);
    H.deferred_free.clear();
  }
  if (f32 && pw32)
    for (int k = 1; k <= H.coarsest; ++k) { H.pool.free(H.L[k].S64); H.L[k].S64 = nullptr; }
  return FEB_OK;
}

// a bounded wait inside the tensor-core K.u gave up (the kernel skipped its work and returned)
int check_tc_status(FebHandle* h) {
  if (!h->tc_status) return FEB_OK;
  int st = 0;
  FEB_CUDA(cudaMemcpyAsync(&st, h->tc_status, sizeof(int), cudaMemcpyDeviceToHost, h->s));
  FEB_CUDA(cudaStreamSynchronize(h->s));
  if (st) { set_last_error("tensor-core K.u: an mbarrier wait timed out"); return FEB_ERR_TIMEOUT; }
  return FEB_OK;
}

// The device's default stream-ordered pool serves every allocation of a handle.  Freed memory stays mapped
// (release threshold at its maximum) for the next handle, and the pool is reserved up front in one block of
// about twice the largest set-up seen (at least ~3 KB per node): growing it piece by piece during set-up
// costs up to hundreds of milliseconds per new peak, in whichever stage happens to need the memory.  The
// used-memory peak drifts a little from one set-up to the next (whether a block freed on one stream is
// reused by another depends on timing), so the pool is grown only on a real shortage, reserved memory below
// 1.25 x that peak or below the size estimate, not whenever the peak passes half of the reservation.
std::atomic<int> g_pool_grows{0};

void reserve_pool(int64_t nnode, int64_t nnode_total, cudaStream_t caller) {
  int dev = 0;
  cudaMemPool_t mp;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetDefaultMemPool(&mp, dev) != cudaSuccess) return;
  uint64_t keep = UINT64_MAX;
  cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &keep);
  uint64_t have = 0, high = 0;
  cudaMemPoolGetAttribute(mp, cudaMemPoolAttrReservedMemCurrent, &have);
  cudaMemPoolGetAttribute(mp, cudaMemPoolAttrUsedMemHigh, &high);
  const uint64_t nodes = (uint64_t)std::max(nnode, nnode_total);
  if (have >= std::max<uint64_t>(high + high / 4, nodes * 3072ull)) return;
  uint64_t want = std::max<uint64_t>(2 * high, nodes * 3072ull);
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) want = std::min<uint64_t>(want, have + free_b / 2);
  if (have >= want) return;
  // the pool serves a request from its free reserved memory first: to hold `want` it must be asked for all of it
  // beyond what is in use now
  uint64_t used = 0;
  cudaMemPoolGetAttribute(mp, cudaMemPoolAttrUsedMemCurrent, &used);
  if (used >= want) return;
  void* p = nullptr;
  const auto t0 = std::chrono::steady_clock::now();
  if (cudaMallocAsync(&p, want - used, caller) == cudaSuccess) {
    cudaFreeAsync(p, caller);
    cudaStreamSynchronize(caller);      // the block is free for the handle's own stream from here on
    // the reservation itself must not count as a set-up's peak (the next handle would double it again)
    uint64_t reset = 0;
    cudaMemPoolSetAttribute(mp, cudaMemPoolAttrUsedMemHigh, &reset);
    g_pool_grows.fetch_add(1);
  }
  cudaGetLastError();                   // a failed reservation is not an error: set-up grows the pool as needed
  if (std::getenv("FEB_POOL_LOG"))      // FEB_POOL_LOG=1: every growth on stderr (diagnostics)
    std::fprintf(stderr, "feb pool: reserved %.2f -> %.2f GB (used peak %.2f GB) in %.2f ms\n", have / 1e9,
                 want / 1e9, high / 1e9,
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
}

int env_flag(const char* name) {
  const char* v = std::getenv(name);
  return v && *v && std::strcmp(v, "0") != 0;
}

// the parts of FebInfo that describe the handle (hierarchy, smoother estimates, kernel shapes, set-up times)
int fill_handle_info(FebHandle& H, FebInfo& inf) {
  inf.t_setup_ms = H.t_setup_ms;
  inf.levels = H.coarsest + 1;
  inf.ndof = H.ndof;
  inf.coarse_n = H.nd;
  std::vector<LevelParams> lp(kMaxLevels);
  FEB_CUDA(cudaMemcpyAsync(lp.data(), H.lp, kMaxLevels * sizeof(LevelParams), cudaMemcpyDeviceToHost, H.s));
  FEB_CUDA(cudaStreamSynchronize(H.s));
  for (int l = 0; l <= H.coarsest && l < 8; ++l) {
    inf.level_dofs[l] = H.L[l].ndof;
    inf.lmax[l] = l < H.coarsest ? lp[l].lmax : 0.0;
  }
  inf.kernel_launches = H.launches;
  for (int i = 0; i < 7; ++i) inf.t_stage_ms[i] = H.stage_ms[i];
  inf.t_stage_ms[7] = H.t_pre_ms;
  inf.ku_shape[0] = H.ku32.tc ? 0 : H.ku32.ty; inf.ku_shape[1] = H.ku32.zchunk;
  inf.ku_shape[2] = H.ku64.ty; inf.ku_shape[3] = H.ku64.zchunk;
  inf.ku_kind = (H.tc_ok && H.ku32.tc) ? 2 : (H.pair_ok ? 1 : 0);
  if (H.pair_ok) {
    if (!(H.tc_ok && H.ku32.tc)) { inf.ku_shape[0] = H.pc32.wy; inf.ku_shape[1] = H.pc32.zchunk; }
    inf.ku_shape[2] = H.pc64.wy; inf.ku_shape[3] = H.pc64.zchunk;
  }
  return FEB_OK;
}

// One instance of a batched solve as three pieces of graph G: the start (device-side stop threshold from ||f||,
// the start vector, ||r0||), a device-side while loop of CG iterations (the loop's condition is the instance's
// own convergence flag), and the finish (result copy, true residual, state read-back into pinned memory).
int add_batch_instance(FebHandle& H, cudaGraph_t G, const double* f_in, const double* x0_in, double* xout,
                       double tol) {
  const int64_t n = 3 * H.ntotal;
  const bool mixed = H.opt.precision != FEB_PREC_FP64;
  CgState init{};
  init.tol2 = tol * tol;
  init.maxiter = H.opt.maxiter;
  *H.st_h = init;   // read by the graph's first node when the graph runs
  // start
  cudaGraph_t pre = nullptr;
  FEB_CUDA(cudaStreamBeginCapture(H.s, cudaStreamCaptureModeThreadLocal));
  FEB_CUDA(cudaMemcpyAsync(H.st, H.st_h, sizeof(CgState), cudaMemcpyHostToDevice, H.s));
  k_masked_copy<<<div_up(n, kThreads), kThreads, 0, H.s>>>(f_in, H.L[0].used, H.ntotal, H.fb);
  launch_dot_partial<double, double>(H.fb, H.fb, n, H.partials, nullptr, H.s);
  launch_finalize(FIN_THR, H.partials, H.st, nullptr, 0, nullptr, H.s);
  if (x0_in) {
    k_masked_copy<<<div_up(n, kThreads), kThreads, 0, H.s>>>(x0_in, H.L[0].used, H.ntotal, H.x);
    H.apply<double>(0, H.x, H.q, nullptr);
    launch_residual<double>(H.fb, H.q, H.r, n, nullptr, H.s);
  } else {
    FEB_CUDA(cudaMemsetAsync(H.x, 0, n * sizeof(double), H.s));
    FEB_CUDA(cudaMemcpyAsync(H.r, H.fb, n * sizeof(double), cudaMemcpyDeviceToDevice, H.s));
  }
  launch_dot_partial<double, double>(H.r, H.r, n, H.partials, nullptr, H.s);
  launch_finalize(FIN_INIT, H.partials, H.st, nullptr, 0, nullptr, H.s);
  if (mixed) launch_convert<double, float>(H.r, H.rf, n, nullptr, H.s);
  FEB_CUDA(cudaStreamEndCapture(H.s, &pre));
  cudaGraphNode_t npre, ncond, npost;
  FEB_CUDA(cudaGraphAddChildGraphNode(&npre, G, nullptr, 0, pre));
  FEB_CUDA(cudaGraphDestroy(pre));
  // iterations
  cudaGraphConditionalHandle cond;
  FEB_CUDA(cudaGraphConditionalHandleCreate(&cond, G, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  FEB_CUDA(cudaGraphAddNode(&ncond, G, &npre, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  FEB_CUDA(cudaStreamBeginCaptureToGraph(H.s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  H.cg_body<double>(H.st, H.x, H.r, H.z, H.p, H.q);
  launch_set_condition(cond, H.st, H.s);
  FEB_CUDA(cudaStreamEndCapture(H.s, &body));
  // finish
  cudaGraph_t post = nullptr;
  FEB_CUDA(cudaStreamBeginCapture(H.s, cudaStreamCaptureModeThreadLocal));
  FEB_CUDA(cudaMemcpyAsync(xout, H.x, n * sizeof(double), cudaMemcpyDeviceToDevice, H.s));
  H.apply<double>(0, xout, H.q, nullptr);
  launch_residual<double>(H.fb, H.q, H.r, n, nullptr, H.s);
  launch_dot_partial<double, double>(H.r, H.r, n, H.partials, nullptr, H.s);
  launch_finalize(FIN_TRUE, H.partials, H.st, nullptr, 0, nullptr, H.s);
  FEB_CUDA(cudaMemcpyAsync(H.st_h, H.st, sizeof(CgState), cudaMemcpyDeviceToHost, H.s));
  FEB_CUDA(cudaStreamEndCapture(H.s, &post));
  FEB_CUDA(cudaGraphAddChildGraphNode(&npost, G, &ncond, 1, post));
  FEB_CUDA(cudaGraphDestroy(post));
  return FEB_OK;
}

}  // namespace
}  // namespace feb

// ================================================================================================== C ABI
extern "C" {

const char* feb_last_error(void) { return g_err; }

void feb_default_options(FebOptions* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = FEB_PREC_FP64;
  o->maxiter = 800;
  o->tol = 1e-6;
  o->min_dofs = 6000;
  o->max_levels = 6;
  o->cheb_degree = 3;
  o->check_every = 1;
  o->inner_tol = 1e-3;
  o->inner_maxiter = 200;
  o->use_graphs = 2;
  o->seed = 0;
  o->x0_mode = 2;
  o->level_kernel = 0;
}

int feb_create(const FebGrid* grid, const FebOperator* op, const FebOptions* opt, void* stream, FebHandle** out) {
  if (!grid || !op || !out || !grid->xe || !grid->ye || !grid->ze || !op->mat || !op->active) {
    set_last_error("feb_create: null argument");
    return FEB_ERR_ARG;
  }
  *out = nullptr;
  if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1) { set_last_error("feb_create: empty grid"); return FEB_ERR_ARG; }
  if (op->mat_mode < 0 || op->mat_mode > 2) { set_last_error("feb_create: bad mat_mode"); return FEB_ERR_ARG; }
  const auto t_entry = std::chrono::steady_clock::now();
  reserve_pool((int64_t)(grid->nx + 1) * (grid->ny + 1) * (grid->nz + 1), op->nnode_total, (cudaStream_t)stream);
  FebHandle* h = new FebHandle((cudaStream_t)stream);
  if (opt) h->opt = *opt; else feb_default_options(&h->opt);
  if (h->opt.cheb_degree < 1 || h->opt.cheb_degree > 9) { delete h; set_last_error("cheb_degree must be 1..9"); return FEB_ERR_ARG; }
  h->mode = op->mat_mode;
  h->nx = grid->nx; h->ny = grid->ny; h->nz = grid->nz;
  h->xe.assign(grid->xe, grid->xe + grid->nx + 1);
  h->ye.assign(grid->ye, grid->ye + grid->ny + 1);
  h->ze.assign(grid->ze, grid->ze + grid->nz + 1);
  h->nnode = (int64_t)(grid->nx + 1) * (grid->ny + 1) * (grid->nz + 1);
  h->ntotal = op->nnode_total > 0 ? op->nnode_total : h->nnode;
  if (h->ntotal < h->nnode || h->ntotal > INT32_MAX / 3) { delete h; set_last_error("feb_create: bad nnode_total"); return FEB_ERR_ARG; }
  h->ev0 = g_streams.event();
  h->ev1 = g_streams.event();
  for (auto& e : h->stage_ev) e = g_streams.event();
  if (!h->s || !h->ev_sync || !h->ev0 || !h->ev1) { delete h; set_last_error("feb_create: stream / event creation failed"); return FEB_ERR_CUDA; }
  if (h->sync_in() != FEB_OK) { delete h; return FEB_ERR_CUDA; }
  cudaEventRecord(h->ev0, h->s);
  h->t_pre_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_entry).count();
  h->stage_mark();   // 0: start
  g_prof.start(env_flag("FEB_PROFILE_SETUP") != 0);
  int st = FEB_OK;
  do {
    h->L.reserve(kMaxLevels);
    h->L.emplace_back();
    if ((st = h->pool.alloc(&h->lp, kMaxLevels)) != FEB_OK) break;
    if ((st = h->pool.zeros(&h->st, 1)) != FEB_OK) break;
    if ((st = h->pool.zeros(&h->sti, 1)) != FEB_OK) break;
    if ((st = h->pool.alloc(&h->partials, kRedBlocks)) != FEB_OK) break;
    if ((st = h->pool.zeros(&h->ctr, 4)) != FEB_OK) break;
    if ((st = h->pool.zeros(&h->sc, 4)) != FEB_OK) break;
    if ((st = h->pool.zeros(&h->status, 1)) != FEB_OK) break;
    if (!(h->st_h = g_pinned.take())) { st = FEB_ERR_CUDA; set_last_error("cudaMallocHost"); break; }
    st = (h->mode == MAT_ORTHO) ? setup_level0<6>(h, op) : setup_level0<2>(h, op);
    if (st != FEB_OK) break;
    st = build_hierarchy(h);
    if (st != FEB_OK) break;
    const size_t n = 3 * (size_t)h->ntotal;
    if ((st = h->pool.zeros(&h->x, n)) != FEB_OK) break;
    if ((st = h->pool.zeros(&h->r, n)) != FEB_OK) break;
    if ((st = h->pool.zeros(&h->z, n)) != FEB_OK) break;
    if ((st = h->pool.zeros(&h->p, n)) != FEB_OK) break;
    if ((st = h->pool.zeros(&h->q, n)) != FEB_OK) break;
    if ((st = h->pool.zeros(&h->fb, n)) != FEB_OK) break;
    if (h->opt.precision != FEB_PREC_FP64) {
      if ((st = h->pool.zeros(&h->xf, n)) != FEB_OK) break;
      if ((st = h->pool.zeros(&h->rf, n)) != FEB_OK) break;
      if ((st = h->pool.zeros(&h->zf, n)) != FEB_OK) break;
      if ((st = h->pool.zeros(&h->pf, n)) != FEB_OK) break;
      if ((st = h->pool.zeros(&h->qf, n)) != FEB_OK) break;
    }
    h->pool.free(h->mat_all);
    h->mat_all = nullptr;
  } while (0);
  if (st == FEB_OK) {
    cudaEventRecord(h->ev1, h->s);
    if (cudaEventSynchronize(h->ev1) != cudaSuccess) { st = FEB_ERR_CUDA; set_last_error("feb_create: %s", cudaGetErrorString(cudaGetLastError())); }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->t_setup_ms = ms;
    for (int i = 0; i + 1 < h->stage_n; ++i) {
      float t = 0.f;
      cudaEventElapsedTime(&t, h->stage_ev[i], h->stage_ev[i + 1]);
      h->stage_ms[i] = t;
    }
  }
  if (st != FEB_OK) {
    delete h;
    return st;
  }
  g_prof.mark("work vectors", h->s);
  g_prof.print();
  h->sync_out();
  *out = h;
  return FEB_OK;
}

int feb_set_rigid_groups(FebHandle* h, int32_t ngroups, const int64_t* offsets, const int64_t* nodes) {
  if (!h || ngroups < 0 || (ngroups > 0 && (!offsets || !nodes))) { set_last_error("feb_set_rigid_groups: bad argument"); return FEB_ERR_ARG; }
  FebHandle& H = *h;
  FEB_TRY(H.sync_in());
  H.has_rigid = false;
  if (H.g_outer) { cudaGraphExecDestroy(H.g_outer); H.g_outer = nullptr; }
  if (H.g_inner) { cudaGraphExecDestroy(H.g_inner); H.g_inner = nullptr; }
  if (ngroups == 0) return FEB_OK;
  // keep used nodes of every group, drop groups with fewer than 4 (rb/splitfe.py:105-112); the filtering and
  // the compaction run on the device, the host sees the per-group counts only
  std::vector<int64_t> off_in(offsets, offsets + ngroups + 1);
  int64_t maxlen = 0;
  for (int g = 0; g < ngroups; ++g) {
    if (off_in[g + 1] < off_in[g]) { set_last_error("feb_set_rigid_groups: offsets decrease at group %d", g); return FEB_ERR_ARG; }
    maxlen = std::max(maxlen, off_in[g + 1] - off_in[g]);
  }
  const int nchunk = (int)std::max<int64_t>(1, (maxlen + 1023) / 1024);
  const dim3 ggrid(nchunk, std::min(ngroups, 65535));
  int64_t* d_off_in = nullptr;
  int *d_count = nullptr, *d_dst = nullptr, *d_chunk = nullptr;
  FEB_TRY(H.pool.upload(&d_off_in, off_in.data(), off_in.size()));
  FEB_TRY(H.pool.zeros(&d_count, (size_t)ngroups + 1));     // counts, then the out-of-range flag
  FEB_TRY(H.pool.alloc(&d_chunk, (size_t)ngroups * nchunk));
  k_group_count<<<ggrid, 1024, 0, H.s>>>(nodes, d_off_in, H.L[0].used, H.ntotal, ngroups, nchunk, d_chunk, d_count,
                                         d_count + ngroups);
  note_launch();
  std::vector<int> cnt(ngroups + 1);
  FEB_CUDA(cudaMemcpyAsync(cnt.data(), d_count, cnt.size() * sizeof(int), cudaMemcpyDeviceToHost, H.s));
  FEB_CUDA(cudaStreamSynchronize(H.s));
  if (cnt[ngroups]) { set_last_error("feb_set_rigid_groups: a group node is out of range"); return FEB_ERR_ARG; }
  std::vector<int> off(1, 0), dst(ngroups, -1);
  for (int g = 0; g < ngroups; ++g) {
    if (cnt[g] < 4) continue;
    dst[g] = off.back();
    off.push_back(off.back() + cnt[g]);
  }
  const int G = (int)off.size() - 1;
  if (G == 0) return FEB_OK;
  const int64_t nkept = off.back();
  int* doff;
  int64_t* dnodes;
  double* cen;
  FEB_TRY(H.pool.upload(&d_dst, dst.data(), dst.size()));
  FEB_TRY(H.pool.upload(&doff, off.data(), off.size()));
  FEB_TRY(H.pool.alloc(&dnodes, (size_t)nkept));
  k_group_compact<<<ggrid, 1024, 0, H.s>>>(nodes, d_off_in, H.L[0].used, ngroups, nchunk, d_chunk, d_dst, dnodes);
  note_launch();
  FEB_TRY(H.pool.alloc(&cen, 3 * (size_t)G));
  RigidView& Z = H.Z;
  Z.ngroups = G; Z.off = doff; Z.nodes = dnodes; Z.cen = cen;
  Z.nxn = H.nx + 1; Z.nyn = H.ny + 1; Z.nnode = H.nnode; Z.orig_copy = H.orig_copy;
  Z.xe = H.xe_d; Z.ye = H.ye_d; Z.ze = H.ze_d;
  const int nc = 6 * G;
  FEB_TRY(H.pool.alloc(&H.zpart, (size_t)rigid_blocks(Z) * G * 6));
  launch_centroids(Z, cen, H.zpart, H.s);
  double* rho = nullptr;
  FEB_TRY(H.pool.alloc(&rho, 3 * (size_t)nkept));
  Z.rho = rho;
  launch_rigid_rho(Z, rho, H.s);
  FEB_TRY(H.pool.alloc(&H.zr, nc));
  FEB_TRY(H.pool.alloc(&H.zcoef, nc));
  // Ec = Z^T K Z column by column (FP64 matrix-free K); the columns stay on the device until one read-back
  std::vector<double> Ec((size_t)nc * nc);
  double *col, *kcol, *Ecd;
  FEB_TRY(H.pool.alloc(&col, 3 * (size_t)H.ntotal));
  FEB_TRY(H.pool.alloc(&kcol, 3 * (size_t)H.ntotal));
  FEB_TRY(H.pool.alloc(&Ecd, (size_t)nc * nc));
  FEB_TRY(H.wait_fine());
  if (!H.rs) {
    H.rs = g_streams.stream();
    if (!H.rs_fork) H.rs_fork = g_streams.event();
    if (!H.rs_join) H.rs_join = g_streams.event();
    if (!H.rs || !H.rs_fork || !H.rs_join) { set_last_error("feb_set_rigid_groups: stream / event creation failed"); return FEB_ERR_CUDA; }
  }
  for (int c = 0; c < nc; ++c) {
    FEB_CUDA(cudaMemsetAsync(col, 0, 3 * (size_t)H.ntotal * sizeof(double), H.s));
    launch_z_column(Z, c, col, H.s);
    H.apply<double>(0, col, kcol, nullptr);
    launch_ztr(Z, kcol, H.zpart, H.zr, H.s);
    FEB_CUDA(cudaMemcpyAsync(Ecd + (size_t)c * nc, H.zr, nc * sizeof(double), cudaMemcpyDeviceToDevice, H.s));
  }
  // while the device forms the columns: the solve's iteration graph, with the rigid-mode correction (its
  // pseudo-inverse is written into Einv below, before any solve reads it)
  FEB_TRY(H.pool.alloc(&H.Einv, (size_t)nc * nc));
  H.has_rigid = true;
  auto undo = [&](int code) {            // no rigid correction, and no graph that applies one
    H.has_rigid = false;
    if (H.g_outer) { cudaGraphExecDestroy(H.g_outer); H.g_outer = nullptr; }
    if (H.g_inner) { cudaGraphExecDestroy(H.g_inner); H.g_inner = nullptr; }
    return code;
  };
  if (const int cst = H.prepare_graphs(); cst != FEB_OK) return undo(cst);
  FEB_CUDA(cudaMemcpyAsync(Ec.data(), Ecd, Ec.size() * sizeof(double), cudaMemcpyDeviceToHost, H.s));
  FEB_CUDA(cudaStreamSynchronize(H.s));
  H.pool.free(col);
  H.pool.free(kcol);
  H.pool.free(Ecd);
  H.pool.free(d_off_in);
  H.pool.free(d_count);
  H.pool.free(d_dst);
  H.pool.free(d_chunk);
  std::vector<double> Es((size_t)nc * nc);
  for (int i = 0; i < nc; ++i)
    for (int j = 0; j < nc; ++j) Es[(size_t)i * nc + j] = 0.5 * (Ec[(size_t)i * nc + j] + Ec[(size_t)j * nc + i]);
  std::vector<double> Ei = sym_pinv(Es, nc);
  if (const int cst = g_staging.copy(H.Einv, Ei.data(), Ei.size() * sizeof(double), H.s); cst != FEB_OK)
    return undo(cst);
  return H.sync_out();
}

int feb_solve(FebHandle* h, const double* f, const double* x0, double* xout, FebInfo* info) {
  if (!h || !f || !xout) { set_last_error("feb_solve: null argument"); return FEB_ERR_ARG; }
  static int fail_once_used = 0;
  if (env_flag("FEB_TEST_FAIL")) { set_last_error("injected failure (FEB_TEST_FAIL)"); return FEB_ERR_INJECTED; }
  if (env_flag("FEB_TEST_FAIL_ONCE") && !fail_once_used) {
    fail_once_used = 1;
    set_last_error("injected transient failure (FEB_TEST_FAIL_ONCE)");
    return FEB_ERR_INJECTED;
  }
  FebHandle& H = *h;
  if (H.coarsest < 0) { set_last_error("feb_solve: handle built with max_levels = 0 (operator only)"); return FEB_ERR_ARG; }
  const int64_t n = 3 * H.ntotal;
  FEB_TRY(H.settle());
  FEB_TRY(H.sync_in());
  H.launches = 0;
  FebInfo inf{};
  FEB_CUDA(cudaEventRecord(H.ev0, H.s));
  // loads and start values on nodes no active cell uses are dropped (fe/solver.py:216-219)
  k_masked_copy<<<div_up(n, kThreads), kThreads, 0, H.s>>>(f, H.L[0].used, H.ntotal, H.fb); note_launch();
  f = H.fb;
  if (x0) {
    k_masked_copy<<<div_up(n, kThreads), kThreads, 0, H.s>>>(x0, H.L[0].used, H.ntotal, H.z); note_launch();
    x0 = H.z;
  }
  int st = FEB_OK;
  int err = FEB_OK;
  const double fn2 = H.read_dot(f, f, n, &err);
  if (err) return err;
  const double fnorm = std::sqrt(fn2);
  const double thr2 = fn2 > 0 ? H.opt.tol * H.opt.tol * fn2 : 1.0;
  // Start value.  x0_mode 2 (default): s = x0 + M (f - K x0), one application of the preconditioner, which
  // removes the start's rough (high-frequency) error; modes 1-2 then use a s with a = s.f / s.K s, the multiple of s
  // closest to the solution in the energy norm (||x* - a s||_K^2 = ||x*||_K^2 - (s.f)^2 / s.K s, never above the
  // zero start's error); when s.f <= 0 the solve starts from zero.  Mode 0 uses x0 as given.
  inf.x0_scale = 0.f;
  if (x0 && fn2 > 0.0 && H.opt.x0_mode >= 1) {
    if (H.opt.x0_mode >= 2) {
      H.apply<double>(0, H.z, H.q, nullptr);
      launch_residual<double>(f, H.q, H.r, n, nullptr, H.s);
      H.precondition<double>(H.r, H.p, nullptr);
      k_axpy_inplace<<<div_up(n, kThreads), kThreads, 0, H.s>>>(H.z, H.p, n, 1.0); note_launch();
    }
    H.apply<double>(0, H.z, H.q, nullptr);
    const double sf = H.read_dot(H.z, f, n, &err);
    if (err) return err;
    const double sks = H.read_dot(H.z, H.q, n, &err);
    if (err) return err;
    if (sf > 0.0 && sks > 0.0 && std::isfinite(sf) && std::isfinite(sks)) {
      const double a = sf / sks;
      k_axpy_inplace<<<div_up(n, kThreads), kThreads, 0, H.s>>>(H.z, H.z, n, a - 1.0); note_launch();
      inf.x0_scale = (float)a;
    } else {
      x0 = nullptr;
    }
  } else if (x0) {
    inf.x0_scale = 1.f;
  }
  inf.x0_used = x0 ? 1 : 0;
  if (fn2 == 0.0) {
    FEB_CUDA(cudaMemsetAsync(xout, 0, n * sizeof(double), H.s));
    inf.flag = 0; inf.iters = 0; inf.relres = 0.0;
  } else if (H.opt.precision != FEB_PREC_REFINE) {
    if (x0) FEB_CUDA(cudaMemcpyAsync(H.x, x0, n * sizeof(double), cudaMemcpyDeviceToDevice, H.s));
    FEB_TRY(H.cg_start<double>(H.st, f, H.x, H.r, x0 != nullptr, thr2, H.opt.maxiter));
    CgState out{};
    FEB_TRY(H.run_cg(H.st, false, out));
    inf.iters = out.it; inf.flag = out.flag; inf.sweeps = 1;
    st = out.status;
    FEB_CUDA(cudaMemcpyAsync(xout, H.x, n * sizeof(double), cudaMemcpyDeviceToDevice, H.s));
  } else {
    // FP64 iterative refinement: r = f - K x (FP64), e = FP32 GMG-PCG(r / ||r||), x += ||r|| e
    if (x0) FEB_CUDA(cudaMemcpyAsync(H.x, x0, n * sizeof(double), cudaMemcpyDeviceToDevice, H.s));
    else FEB_CUDA(cudaMemsetAsync(H.x, 0, n * sizeof(double), H.s));
    int total = 0, sweeps = 0;
    inf.flag = H.opt.maxiter;
    for (; sweeps < 1000; ++sweeps) {
      H.apply<double>(0, H.x, H.q, nullptr);
      launch_residual<double>(f, H.q, H.r, n, nullptr, H.s);
      double rr = H.read_dot(H.r, H.r, n, &err);
      if (err) return err;
      if (!std::isfinite(rr)) { st = FEB_ERR_NAN; break; }
      if (rr < thr2) { inf.flag = 0; break; }
      if (total >= H.opt.maxiter) break;
      double scale[2] = {std::sqrt(rr), 1.0 / std::sqrt(rr)};
      FEB_CUDA(cudaMemcpyAsync(H.sc, scale, 2 * sizeof(double), cudaMemcpyHostToDevice, H.s));
      launch_scale_to_float(H.r, H.rf, H.sc + 1, n, nullptr, H.s);
      // the inner CG starts from r32 as its right-hand side (stored in qf's partner pf? use bf = zf temp)
      FEB_CUDA(cudaMemcpyAsync(H.L[0].b32, H.rf, n * sizeof(float), cudaMemcpyDeviceToDevice, H.s));
      int budget = std::min(H.opt.inner_maxiter, H.opt.maxiter - total);
      FEB_TRY(H.cg_start<float>(H.sti, H.L[0].b32, H.xf, H.rf, false, H.opt.inner_tol * H.opt.inner_tol, budget));
      CgState out{};
      FEB_TRY(H.run_cg(H.sti, true, out));
      total += out.it;
      if (out.status == FEB_ERR_NAN) { st = FEB_ERR_NAN; break; }
      launch_add_scaled(H.xf, H.x, H.sc, n, nullptr, H.s);
      H.launches += 6;
      if (out.it == 0) break;
    }
    inf.iters = total; inf.sweeps = sweeps + 1;
    FEB_CUDA(cudaMemcpyAsync(xout, H.x, n * sizeof(double), cudaMemcpyDeviceToDevice, H.s));
  }
  // true FP64 residual of the result
  if (fn2 > 0) {
    H.apply<double>(0, xout, H.q, nullptr);
    launch_residual<double>(f, H.q, H.r, n, nullptr, H.s);
    double rr = H.read_dot(H.r, H.r, n, &err);
    if (err) return err;
    inf.relres = std::sqrt(rr) / fnorm;
  }
  FEB_CUDA(cudaEventRecord(H.ev1, H.s));
  FEB_CUDA(cudaEventSynchronize(H.ev1));
  FEB_TRY(check_tc_status(h));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, H.ev0, H.ev1);
  inf.t_solve_ms = ms;
  FEB_TRY(fill_handle_info(H, inf));
  if (info) *info = inf;
  FEB_TRY(H.sync_out());
  if (st != FEB_OK) {
    set_last_error(st == FEB_ERR_BREAKDOWN ? "CG breakdown: p^T K p <= 0" : "non-finite residual");
    return st;
  }
  return FEB_OK;
}

int feb_solve_batch(FebHandle* const* hs, int32_t n, const double* const* f, const double* const* x0,
                    double* const* x, FebInfo* info) {
  if (!hs || n < 0 || (n > 0 && (!f || !x))) { set_last_error("feb_solve_batch: bad argument"); return FEB_ERR_ARG; }
  if (n == 0) return FEB_OK;
  for (int i = 0; i < n; ++i) {
    if (!hs[i] || !f[i] || !x[i]) { set_last_error("feb_solve_batch: null handle or vector at %d", i); return FEB_ERR_ARG; }
    if (hs[i]->coarsest < 0) { set_last_error("feb_solve_batch: handle %d built with max_levels = 0", i); return FEB_ERR_ARG; }
    if (hs[i]->opt.precision == FEB_PREC_REFINE) {
      set_last_error("feb_solve_batch: handle %d uses the refined precision (host-driven sweeps); use feb_solve", i);
      return FEB_ERR_ARG;
    }
    for (int j = 0; j < i; ++j)
      if (hs[j] == hs[i]) { set_last_error("feb_solve_batch: handle %d given twice", i); return FEB_ERR_ARG; }
  }
  for (int i = 0; i < n; ++i) FEB_TRY(hs[i]->settle());
  FebHandle& H0 = *hs[0];
  const long long before = g_launches.load();
  cudaGraph_t G = nullptr;
  cudaGraphExec_t ex = nullptr;
  int st = FEB_OK;
  auto fail = [&](int code) {
    if (ex) cudaGraphExecDestroy(ex);
    if (G) cudaGraphDestroy(G);
    g_launches.store(before);
    return code;
  };
  if (cudaGraphCreate(&G, 0) != cudaSuccess) { set_last_error("cudaGraphCreate"); return FEB_ERR_CUDA; }
  for (int i = 0; i < n; ++i) {
    FebHandle& H = *hs[i];
    if ((st = H.sync_in()) != FEB_OK) return fail(st);
    if ((st = add_batch_instance(H, G, f[i], x0 ? x0[i] : nullptr, x[i], H.opt.tol)) != FEB_OK) return fail(st);
  }
  g_launches.store(before);   // captured kernels are counted below, once per run
  if (cudaGraphInstantiate(&ex, G, 0) != cudaSuccess) { set_last_error("feb_solve_batch: graph instantiation failed"); return fail(FEB_ERR_CUDA); }
  // every instance's stream has reached its inputs (sync_in); the batch runs on instance 0's stream after all
  for (int i = 1; i < n; ++i) {
    if (cudaEventRecord(hs[i]->ev_sync, hs[i]->s) != cudaSuccess ||
        cudaStreamWaitEvent(H0.s, hs[i]->ev_sync, 0) != cudaSuccess) { set_last_error("feb_solve_batch: stream join"); return fail(FEB_ERR_CUDA); }
  }
  cudaEventRecord(H0.ev0, H0.s);
  if (cudaGraphLaunch(ex, H0.s) != cudaSuccess) { set_last_error("feb_solve_batch: graph launch failed"); return fail(FEB_ERR_CUDA); }
  cudaEventRecord(H0.ev1, H0.s);
  if (cudaEventSynchronize(H0.ev1) != cudaSuccess) {
    set_last_error("feb_solve_batch: %s", cudaGetErrorString(cudaGetLastError()));
    return fail(FEB_ERR_CUDA);
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, H0.ev0, H0.ev1);
  int first_err = FEB_OK;
  for (int i = 0; i < n; ++i) {
    FebHandle& H = *hs[i];
    const CgState S = *H.st_h;
    FebInfo inf{};
    inf.iters = S.it; inf.flag = S.flag; inf.sweeps = 1;
    inf.relres = S.fn2 > 0 ? std::sqrt(S.rtrue / S.fn2) : 0.0;
    inf.t_solve_ms = ms;    // the whole batch: the instances run concurrently
    inf.x0_used = x0 && x0[i] ? 1 : 0;
    inf.x0_scale = inf.x0_used ? 1.f : 0.f;
    H.launches = 0;
    if ((st = fill_handle_info(H, inf)) != FEB_OK) return fail(st);
    if (info) info[i] = inf;
    if (S.status != FEB_OK && first_err == FEB_OK) first_err = S.status;
    if ((st = H.sync_out()) != FEB_OK) return fail(st);
  }
  if (ex) cudaGraphExecDestroy(ex);
  cudaGraphDestroy(G);
  if (first_err != FEB_OK) {
    set_last_error(first_err == FEB_ERR_BREAKDOWN ? "CG breakdown: p^T K p <= 0" : "non-finite residual");
    return first_err;
  }
  return FEB_OK;
}

int feb_apply(FebHandle* h, int32_t prec, const void* u, void* y) {
  if (!h || !u || !y) { set_last_error("feb_apply: null argument"); return FEB_ERR_ARG; }
  FEB_TRY(h->sync_in());
  FEB_TRY(h->wait_fine());
  if (prec == 0) h->apply<double>(0, (const double*)u, (double*)y, nullptr);
  else h->apply<float>(0, (const float*)u, (float*)y, nullptr);
  FEB_CUDA(cudaGetLastError());
  return h->sync_out();
}

int feb_precondition(FebHandle* h, const double* r, double* z) {
  if (!h || !r || !z) { set_last_error("feb_precondition: null argument"); return FEB_ERR_ARG; }
  if (h->coarsest < 0) { set_last_error("feb_precondition: handle built with max_levels = 0 (operator only)"); return FEB_ERR_ARG; }
  FEB_TRY(h->settle());
  FEB_TRY(h->sync_in());
  h->precondition<double>(r, z, nullptr);
  FEB_CUDA(cudaGetLastError());
  return h->sync_out();
}

int feb_export_solution(FebHandle* h, const double* x, double* U) {
  if (!h || !x || !U) { set_last_error("feb_export_solution: null argument"); return FEB_ERR_ARG; }
  FEB_TRY(h->sync_in());
  k_export<<<div_up(3 * h->ntotal, kThreads), kThreads, 0, h->s>>>(x, h->L[0].used, h->ntotal, U); note_launch();
  FEB_CUDA(cudaGetLastError());
  return h->sync_out();
}

int feb_used_nodes(FebHandle* h, int64_t* nused, uint8_t* mask) {
  if (!h) { set_last_error("feb_used_nodes: null handle"); return FEB_ERR_ARG; }
  if (nused) *nused = h->ndof / 3;
  if (mask) {
    FEB_TRY(h->sync_in());
    FEB_CUDA(cudaMemcpyAsync(mask, h->L[0].used, h->ntotal, cudaMemcpyDeviceToDevice, h->s));
    return h->sync_out();
  }
  return FEB_OK;
}

int feb_benchmark_smooth_set(FebHandle* h, int32_t nbuf, void* const* d, void* const* r, void* const* x,
                             void* const* e, int32_t nrep, float* ms) {
  if (!h || nbuf < 1 || !d || !r || !x || !e || nrep < 1 || !ms) {
    set_last_error("feb_benchmark_smooth_set: bad argument");
    return FEB_ERR_ARG;
  }
  for (int b = 0; b < nbuf; ++b)
    if (!d[b] || !r[b] || !x[b] || !e[b]) { set_last_error("feb_benchmark_smooth_set: null buffer %d", b); return FEB_ERR_ARG; }
  if (h->coarsest < 1 || !h->pair_on<float>()) {
    set_last_error("feb_benchmark_smooth_set: needs a hierarchy and the paired level-0 kernel");
    return FEB_ERR_ARG;
  }
  FEB_TRY(h->settle());     // the Chebyshev coefficients come from the power iteration
  FEB_TRY(h->sync_in());
  FEB_TRY(h->tune_events());
  auto step = [&](int i) {
    const int b = i % nbuf;
    SmoothArgs<float> A;
    A.r_in = (const float*)r[b]; A.r_out = (float*)r[b];
    A.x_in = (const float*)x[b]; A.x_out = (float*)x[b];
    A.d_out = (float*)e[b];
    A.lp = h->lp; A.k = 0;
    h->pair_run<float>((const float*)d[b], nullptr, &A, nullptr);
  };
  step(0);
  FEB_CUDA(cudaEventRecord(h->tev0, h->s));
  for (int i = 0; i < nrep; ++i) step(i);
  FEB_CUDA(cudaEventRecord(h->tev1, h->s));
  FEB_CUDA(cudaEventSynchronize(h->tev1));
  float t = 0.f;
  FEB_CUDA(cudaEventElapsedTime(&t, h->tev0, h->tev1));
  *ms = t / nrep;
  return h->sync_out();
}

int64_t feb_launch_count(void) { return g_launches.load(); }

int feb_pool_stats(int64_t* reserved, int64_t* used_peak, int32_t* grow_events) {
  int dev = 0;
  cudaMemPool_t mp;
  FEB_CUDA(cudaGetDevice(&dev));
  FEB_CUDA(cudaDeviceGetDefaultMemPool(&mp, dev));
  uint64_t have = 0, high = 0;
  FEB_CUDA(cudaMemPoolGetAttribute(mp, cudaMemPoolAttrReservedMemCurrent, &have));
  FEB_CUDA(cudaMemPoolGetAttribute(mp, cudaMemPoolAttrUsedMemHigh, &high));
  if (reserved) *reserved = (int64_t)have;
  if (used_peak) *used_peak = (int64_t)high;
  if (grow_events) *grow_events = g_pool_grows.load();
  return FEB_OK;
}

int feb_benchmark_apply(FebHandle* h, int32_t prec, const void* u, void* y, int32_t nrep, float* ms) {
  if (!h || !u || !y || nrep < 1 || !ms) { set_last_error("feb_benchmark_apply: bad argument"); return FEB_ERR_ARG; }
  FEB_TRY(h->settle());     // the timed products run alone
  FEB_TRY(h->sync_in());
  FEB_CUDA(cudaEventRecord(h->ev0, h->s));
  for (int i = 0; i < nrep; ++i) {
    if (prec == 0) h->apply<double>(0, (const double*)u, (double*)y, nullptr);
    else h->apply<float>(0, (const float*)u, (float*)y, nullptr);
  }
  FEB_CUDA(cudaEventRecord(h->ev1, h->s));
  FEB_CUDA(cudaEventSynchronize(h->ev1));
  float t = 0.f;
  FEB_CUDA(cudaEventElapsedTime(&t, h->ev0, h->ev1));
  *ms = t / nrep;
  FEB_TRY(check_tc_status(h));
  return h->sync_out();
}

int feb_benchmark_apply_set(FebHandle* h, int32_t prec, int32_t nbuf, const void* const* u, void* const* y,
                            int32_t nrep, float* ms) {
  if (!h || nbuf < 1 || !u || !y || nrep < 1 || !ms) {
    set_last_error("feb_benchmark_apply_set: bad argument");
    return FEB_ERR_ARG;
  }
  for (int b = 0; b < nbuf; ++b)
    if (!u[b] || !y[b]) { set_last_error("feb_benchmark_apply_set: null buffer %d", b); return FEB_ERR_ARG; }
  FEB_TRY(h->settle());     // the timed products run alone
  FEB_TRY(h->sync_in());
  FEB_CUDA(cudaEventRecord(h->ev0, h->s));
  for (int i = 0; i < nrep; ++i) {
    const int b = i % nbuf;
    if (prec == 0) h->apply<double>(0, (const double*)u[b], (double*)y[b], nullptr);
    else h->apply<float>(0, (const float*)u[b], (float*)y[b], nullptr);
  }
  FEB_CUDA(cudaEventRecord(h->ev1, h->s));
  FEB_CUDA(cudaEventSynchronize(h->ev1));
  float t = 0.f;
  FEB_CUDA(cudaEventElapsedTime(&t, h->ev0, h->ev1));
  *ms = t / nrep;
  FEB_TRY(check_tc_status(h));
  return h->sync_out();
}

int feb_destroy(FebHandle* h) {
  if (!h) return FEB_OK;
  delete h;
  return FEB_OK;
}

}  // extern "C"
