// batch.cu -- many independent sweep problems in one persistent launch.
//
// The reference sweeps one problem per Sweeper (sweeper_kba_c.h:44-287 sets
// it up, sweeper_kba_c.h:588-845 sweeps it).  A batch takes any number of
// problems of uneven grid, group, angle and moment sizes and sweeps all of
// them in ONE launch of a persistent kernel:
//
//   * Every problem gets the task schedule a Sweeper would build for it
//     (schedule.cpp).  Problems are grouped in classes, one per compiled
//     kernel body (moment count, 32-angle chunks, tile shape); the kernel's
//     CTAs work through the classes in kind order, each class a contiguous
//     range of one task table with global task ids.
//   * The face planes are scratch that a problem needs only while it runs.
//     They come from one arena, placed first-fit in admission order; a problem
//     placed over bytes that earlier problems used waits, on the device, until
//     those problems have completed every task (a per-problem counter).
//   * The order of the table comes from a host-side list-scheduling
//     simulation: one worker per SM, task durations proportional to their
//     wavefront steps, a same-phase neighbour tile released one tile
//     diagonal after its upwind tile starts (the kernel pipelines them plane
//     by plane), other dependencies released at completion, problems admitted
//     while the arena has room.  Tasks enter the table in simulated start
//     order, so dependencies always precede their dependents and the CTAs,
//     which grab tasks in table order, rarely wait.
//   * The reference driver's iteration loop (runner.c:148-155: niterations
//     sweeps, swapping vi and vo) runs as a CUDA graph of one launch per
//     iteration, captured once per iteration count.
//   * The tile shape of each class is chosen by timing both shapes on the
//     class's median problem (autotune), or defaults to 4 x 2.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <queue>
#include <thread>
#include <vector>

#include "internal.h"
#include "sweep_fp64_ws.cuh"

namespace msb {
namespace {

constexpr int kBatchStages = 4;
constexpr long long kBatchTimeoutNs = 4000000000LL;
constexpr size_t kAlign = 256;

inline size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// One entry of the batch: one 32-angle pass of a caller's problem.  A
// problem of na angles has ceil(na / 32) entries; entry c sweeps angles
// [32 c, 32 c + nac) reading the caller's matrices in place, adds to vo from
// the second pass on, uses the first pass's face scratch and starts once the
// pass before it has completed (the order a Sweeper's passes run in, so the
// sums are the same).
struct ProbPlan {
  msb_problem d;
  int user = 0, pass = 0, npass = 1, a0 = 0, nac = 0;
  int prev = -1, next = -1;  // entries of the neighbouring passes
  int nch = 0, ngp = 0, kind = 0, cls = 0, tx = 4, ty = 2;
  Schedule sched;
  size_t face_bytes[3] = {0, 0, 0};
  size_t scratch = 0;      // bytes of the three face arrays
  size_t offset = 0;       // in the arena
  double work = 0.0;       // task steps x relative step cost
  std::vector<int> preds;  // problems whose arena bytes this one reuses
  long long seq = 0;       // admission order
};

struct ClassInfo {
  int kind = 0, nm = 0, nch = 0, tx = 4, ty = 2;
  long long base = 0, ntask = 0;
  double work = 0.0;
};

// relative cost of one wavefront step of a task (one cell column per warp)
double step_cost(int nm, int nch) { return (0.3 + 0.7 * nm / 16.0) * nch; }

}  // namespace

struct BatchImpl {
  std::vector<ProbPlan> probs;  // entries (angle passes of the caller's problems)
  int nuser = 0;                // the caller's problems
  std::vector<ClassInfo> classes;
  int nsm = 0;
  bool device = false;
  size_t arena_bytes = 0;
  // host copies of the table (kept for the host-side checks)
  std::vector<int> rec, task_prob, pred_off, pred, prob_ntask;
  long long ntask = 0;
  double sim_makespan = 0.0;
  double sim_busy = 0.0;  // simulated fraction of worker time spent on tasks
  // device
  void* d_arena = nullptr;
  int* d_tasks = nullptr;
  int* d_task_prob = nullptr;
  Fp64Prob* d_probs = nullptr;
  int* d_pred_off = nullptr;
  int* d_pred = nullptr;
  int* d_prob_ntask = nullptr;
  int* d_sync = nullptr;
  size_t sync_ints = 0;
  long long* d_ptime = nullptr;
  int* h_status = nullptr;
  long long timeout_ns = kBatchTimeoutNs;
  cudaGraphExec_t graph = nullptr;
  int graph_iters = -1;
  cudaStream_t graph_stream = nullptr;
  int launches = 0;

  void free_device() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    cudaFree(d_arena);
    cudaFree(d_tasks);
    cudaFree(d_task_prob);
    cudaFree(d_probs);
    cudaFree(d_pred_off);
    cudaFree(d_pred);
    cudaFree(d_prob_ntask);
    cudaFree(d_sync);
    cudaFree(d_ptime);
    if (h_status) cudaFreeHost(h_status);
    d_arena = nullptr;
    d_tasks = d_task_prob = d_pred_off = d_pred = d_prob_ntask = d_sync = nullptr;
    d_probs = nullptr;
    d_ptime = nullptr;
    h_status = nullptr;
  }
  ~BatchImpl() { free_device(); }
};

namespace {

int check_problem(const msb_problem& p, int i, bool need_ptrs) {
  if (p.ncell_x <= 0 || p.ncell_y <= 0 || p.ncell_z <= 0 || p.ne <= 0 || p.na <= 0)
    return set_error(MSB_ERR_ARG, "batch problem %d: invalid sizes", i);
  if (p.nm != 4 && p.nm != 8 && p.nm != 16)
    return set_error(MSB_ERR_UNSUPPORTED, "batch problem %d: nm %d (4, 8 or 16)", i, p.nm);
  if (p.na > 128) return set_error(MSB_ERR_UNSUPPORTED, "batch problem %d: na %d (a batch takes na <= 128)", i, p.na);
  if (need_ptrs) {
    if (!p.vi || !p.vo || !p.a_from_m || !p.m_from_a)
      return set_error(MSB_ERR_ARG, "batch problem %d: null device pointer", i);
    if (reinterpret_cast<uintptr_t>(p.vi) % 16 || reinterpret_cast<uintptr_t>(p.vo) % 16)
      return set_error(MSB_ERR_ARG, "batch problem %d: state arrays must be 16-byte aligned", i);
  }
  return MSB_OK;
}

// Per-problem schedule and sizes for the given tile of its class.
int plan_problem(ProbPlan& P, int nsm) {
  const msb_problem& d = P.d;
  P.nch = 1;
  P.ngp = (d.ne + 1) / 2;
  // the same task window as a single problem's schedule (4 x SMs)
  const int gpb = pick_gp_block(d.ncell_x, d.ncell_y, P.ngp, P.tx, P.ty, 4 * nsm);
  int rc = build_schedule(d.ncell_x, d.ncell_y, d.ncell_z, P.ngp, P.tx, P.ty, gpb, P.sched);
  if (rc) return rc;
  const size_t per = (size_t)NOCTANT * P.ngp * (size_t)P.nch * 256 * sizeof(double);
  P.face_bytes[0] = align_up(per * d.ncell_y * d.ncell_x);
  P.face_bytes[1] = align_up(per * d.ncell_z * d.ncell_x);
  P.face_bytes[2] = align_up(per * d.ncell_z * d.ncell_y);
  P.scratch = P.face_bytes[0] + P.face_bytes[1] + P.face_bytes[2];
  double steps = 0.0;
  const long long n = P.sched.ntask();
  for (long long t = 0; t < n; ++t) {
    const int* r = &P.sched.rec[t * MSB_TASK_INTS];
    steps += (r[TK_Z1] - r[TK_Z0]) + (r[TK_X1] - r[TK_X0]) + (r[TK_Y1] - r[TK_Y0]) - 2;
  }
  P.work = steps * step_cost(d.nm, P.nch);
  return MSB_OK;
}

// First-fit arena with the last user of every byte range.
struct Arena {
  size_t size;
  std::map<size_t, size_t> free_;           // offset -> length
  std::map<size_t, std::pair<size_t, int>> owner;  // offset -> (length, last problem), disjoint
  explicit Arena(size_t s) : size(s) { free_[0] = s; }
  bool alloc(size_t len, size_t* off) {
    for (auto it = free_.begin(); it != free_.end(); ++it)
      if (it->second >= len) {
        *off = it->first;
        const size_t rest = it->second - len;
        const size_t o2 = it->first + len;
        free_.erase(it);
        if (rest) free_[o2] = rest;
        return true;
      }
    return false;
  }
  void release(size_t off, size_t len) {
    auto it = free_.emplace(off, len).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  // previous owners of [off, off + len); the range then belongs to p
  std::vector<int> take(size_t off, size_t len, int p) {
    std::vector<int> prev;
    const size_t end = off + len;
    auto it = owner.lower_bound(off);
    if (it != owner.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second.first > off) it = pv;
    }
    std::vector<std::pair<size_t, std::pair<size_t, int>>> keep;
    while (it != owner.end() && it->first < end) {
      const size_t a = it->first, b = a + it->second.first;
      const int q = it->second.second;
      prev.push_back(q);
      if (a < off) keep.push_back({a, {off - a, q}});
      if (b > end) keep.push_back({end, {b - end, q}});
      it = owner.erase(it);
    }
    for (auto& k : keep) owner[k.first] = k.second;
    owner[off] = {len, p};
    std::sort(prev.begin(), prev.end());
    prev.erase(std::unique(prev.begin(), prev.end()), prev.end());
    return prev;
  }
};

// Orders every task of the batch (see the file comment).  Fills B.rec,
// task_prob, classes' ranges, offsets and predecessors.
int simulate_and_order(BatchImpl& B) {
  const int np = (int)B.probs.size();
  // admission order: classes in order, problems inside a class by decreasing
  // work
  std::vector<int> order(np);
  for (int i = 0; i < np; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const ProbPlan &A = B.probs[a], &Bp = B.probs[b];
    if (A.cls != Bp.cls) return A.cls < Bp.cls;
    return A.work > Bp.work;
  });
  for (int i = 0; i < np; ++i) B.probs[order[i]].seq = i;
  for (auto& p : B.probs)
    if (p.scratch > B.arena_bytes)
      return set_error(MSB_ERR_ARG, "batch: a problem needs %zu bytes of face scratch, the arena has %zu", p.scratch,
                       B.arena_bytes);

  // global ids of the tasks in problem-major order (the simulation's ids)
  std::vector<long long> first(np + 1, 0);
  for (int p = 0; p < np; ++p) first[p + 1] = first[p] + B.probs[p].sched.ntask();
  const long long N = first[np];
  if (N >= (1LL << 31) - SY_PROGRESS - np - 1) return set_error(MSB_ERR_ARG, "batch: too many tasks (%lld)", N);
  // per task, in one record (the simulation touches them together): its
  // problem, duration, delay until its first plane is through, and the
  // dependencies not yet released
  struct SimTask {
    float dur, plane_delay;
    int left, prob;
  };
  std::vector<SimTask> T(N);
  // dependents, CSR: dcount/dlist released when a task completes, pcount/plist
  // when its first plane is through (a same-phase neighbour's plane-by-plane
  // dependency)
  std::vector<int> dcount(N + 1, 0), pcount(N + 1, 0);
  for (int p = 0; p < np; ++p) {
    const ProbPlan& P = B.probs[p];
    const double c = step_cost(P.d.nm, P.nch);
    for (long long t = 0; t < P.sched.ntask(); ++t) {
      const int* r = &P.sched.rec[t * MSB_TASK_INTS];
      const long long g = first[p] + t;
      T[g].prob = p;
      const int w = r[TK_X1] - r[TK_X0], h = r[TK_Y1] - r[TK_Y0], nz = r[TK_Z1] - r[TK_Z0];
      T[g].dur = (float)(c * (nz + w + h - 2));
      T[g].plane_delay = (float)(c * (w + h - 1));
      int n = 0;
      for (int k = TK_DEP_X; k <= TK_DEP_VO; ++k)
        if (r[k] >= 0) {
          ++n;
          const bool plane = (k == TK_DEP_X && (r[TK_DEP_MODE] & DM_X_PLANE)) ||
                             (k == TK_DEP_Y && (r[TK_DEP_MODE] & DM_Y_PLANE));
          ++(plane ? pcount : dcount)[first[p] + r[k] + 1];
        }
      T[g].left = n;
    }
  }
  for (long long g = 0; g < N; ++g) {
    dcount[g + 1] += dcount[g];
    pcount[g + 1] += pcount[g];
  }
  std::vector<int> dlist(dcount[N]), plist(pcount[N]);
  {
    std::vector<int> fill(dcount.begin(), dcount.end() - 1), pfill(pcount.begin(), pcount.end() - 1);
    for (int p = 0; p < np; ++p) {
      const ProbPlan& P = B.probs[p];
      for (long long t = 0; t < P.sched.ntask(); ++t) {
        const int* r = &P.sched.rec[t * MSB_TASK_INTS];
        const long long g = first[p] + t;
        for (int k = TK_DEP_X; k <= TK_DEP_VO; ++k)
          if (r[k] >= 0) {
            const bool plane = (k == TK_DEP_X && (r[TK_DEP_MODE] & DM_X_PLANE)) ||
                               (k == TK_DEP_Y && (r[TK_DEP_MODE] & DM_Y_PLANE));
            const long long u = first[p] + r[k];
            if (plane)
              plist[pfill[u]++] = (int)g;
            else
              dlist[fill[u]++] = (int)g;
          }
      }
    }
  }

  const int ncls = (int)B.classes.size();
  std::vector<long long> cls_left(ncls, 0);
  for (int p = 0; p < np; ++p) cls_left[B.probs[p].cls] += B.probs[p].sched.ntask();
  std::vector<int> by_seq(np);
  for (int p = 0; p < np; ++p) by_seq[B.probs[p].seq] = p;
  // ready tasks, taken by (admission order, index in the problem's
  // schedule): a min-heap of task ids per problem, and per class a bit per
  // admission slot whose problem has ready tasks
  std::vector<std::priority_queue<long long, std::vector<long long>, std::greater<long long>>> ready(np);
  const int nword = (np + 63) / 64;
  std::vector<std::vector<uint64_t>> has_ready(ncls, std::vector<uint64_t>(nword, 0));
  auto make_ready = [&](long long g) {
    const int p = T[g].prob;
    if (ready[p].empty()) {
      const int q = B.probs[p].seq;
      has_ready[B.probs[p].cls][q >> 6] |= 1ull << (q & 63);
    }
    ready[p].push(g);
  };
  // the next task of class c, or -1
  auto take_ready = [&](int c) -> long long {
    const std::vector<uint64_t>& w = has_ready[c];
    for (int i = 0; i < nword; ++i)
      if (w[i]) {
        const int q = 64 * i + __builtin_ctzll(w[i]);
        const int p = by_seq[q];
        const long long g = ready[p].top();
        ready[p].pop();
        if (ready[p].empty()) has_ready[c][i] &= ~(1ull << (q & 63));
        return g;
      }
    return -1;
  };
  struct Ev {
    double t;
    int kind;  // 0 plane release, 1 finish
    long long g;
    // ties by kind, then task id: the order does not depend on the heap's layout
    bool operator>(const Ev& o) const { return t != o.t ? t > o.t : kind != o.kind ? kind > o.kind : g > o.g; }
  };
  std::priority_queue<Ev, std::vector<Ev>, std::greater<Ev>> ev;
  std::vector<long long> pdone(np, 0);
  Arena arena(B.arena_bytes);
  int next_admit = 0;
  auto push_ready = [&](int p) {
    for (long long t = first[p]; t < first[p + 1]; ++t)
      if (T[t].left == 0) make_ready(t);
  };
  auto admit = [&]() {
    while (next_admit < np) {
      const int p = by_seq[next_admit];
      ProbPlan& P = B.probs[p];
      if (P.prev >= 0) {
        // a later pass: the first pass's scratch, after the pass before it
        P.offset = B.probs[P.prev].offset;
        P.preds = arena.take(P.offset, P.scratch, p);
        if (pdone[P.prev] == B.probs[P.prev].sched.ntask()) push_ready(p);
      } else {
        size_t off = 0;
        if (!arena.alloc(P.scratch, &off)) break;
        P.offset = off;
        P.preds = arena.take(off, P.scratch, p);
        push_ready(p);
      }
      ++next_admit;
    }
  };
  auto release = [&](long long g, bool plane) {
    const std::vector<int>& cnt = plane ? pcount : dcount;
    const std::vector<int>& lst = plane ? plist : dlist;
    for (int k = cnt[g]; k < cnt[g + 1]; ++k)
      if (--T[lst[k]].left == 0) make_ready(lst[k]);
  };

  std::vector<long long> table;
  table.reserve(N);
  int free_w = B.nsm;
  int cur = 0;
  double now = 0.0;
  admit();
  for (;;) {
    while (cur < ncls && cls_left[cur] == 0) ++cur;
    while (free_w > 0 && cur < ncls) {
      const long long g = take_ready(cur);
      if (g < 0) break;
      table.push_back(g);
      --free_w;
      --cls_left[cur];
      ev.push({now + T[g].dur, 1, g});
      if (pcount[g + 1] > pcount[g]) ev.push({now + T[g].plane_delay, 0, g});  // else it releases nothing
      while (cur < ncls && cls_left[cur] == 0) ++cur;
    }
    if (ev.empty()) break;
    const Ev e = ev.top();
    ev.pop();
    now = e.t;
    if (e.kind == 0) {
      release(e.g, true);
    } else {
      ++free_w;
      release(e.g, false);
      const int p = T[e.g].prob;
      if (++pdone[p] == B.probs[p].sched.ntask()) {
        const ProbPlan& P = B.probs[p];
        if (P.next >= 0) {
          if (B.probs[P.next].seq < next_admit) push_ready(P.next);  // admitted, waiting for this pass
        } else {
          arena.release(P.offset, P.scratch);
          admit();
        }
      }
    }
  }
  if ((long long)table.size() != N)
    return set_error(MSB_ERR_ARG, "batch: scheduling simulation left %lld tasks unplaced", N - (long long)table.size());
  B.sim_makespan = now;
  double busy = 0.0;
  for (long long g = 0; g < N; ++g) busy += T[g].dur;
  B.sim_busy = now > 0.0 ? busy / (now * B.nsm) : 0.0;

  // the table in simulated start order, dependencies as global ids
  std::vector<int> pos(N);
  for (long long i = 0; i < N; ++i) pos[table[i]] = (int)i;
  B.ntask = N;
  B.rec.assign((size_t)N * MSB_TASK_INTS, 0);
  B.task_prob.assign(N, 0);
  B.prob_ntask.assign(np, 0);
  {
    // independent records: written by the host's cores in chunks
    std::atomic<bool> bad{false};
    const int nthr = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), 16));
    std::vector<std::thread> pool;
    for (int t = 0; t < nthr; ++t)
      pool.emplace_back([&, t]() {
        const long long i0 = N * t / nthr, i1 = N * (t + 1) / nthr;
        for (long long i = i0; i < i1; ++i) {
          const long long g = table[i];
          const int p = T[g].prob;
          const int* r = &B.probs[p].sched.rec[(g - first[p]) * MSB_TASK_INTS];
          int* o = &B.rec[i * MSB_TASK_INTS];
          std::copy(r, r + MSB_TASK_INTS, o);
          for (int k = TK_DEP_X; k <= TK_DEP_VO; ++k)
            if (r[k] >= 0) {
              o[k] = pos[first[p] + r[k]];
              if (o[k] >= i) bad = true;
            }
          B.task_prob[i] = p;
        }
      });
    for (auto& th : pool) th.join();
    if (bad) return set_error(MSB_ERR_ARG, "batch: table not topological");
  }
  for (int p = 0; p < np; ++p) B.prob_ntask[p] = (int)B.probs[p].sched.ntask();
  for (auto& c : B.classes) c.ntask = 0;
  long long at = 0;
  for (int c = 0; c < ncls; ++c) {
    B.classes[c].base = at;
    while (at < N && B.probs[B.task_prob[at]].cls == c) ++at;
    B.classes[c].ntask = at - B.classes[c].base;
  }
  if (at != N) return set_error(MSB_ERR_ARG, "batch: class ranges are not contiguous");
  B.pred_off.assign(np + 1, 0);
  B.pred.clear();
  for (int p = 0; p < np; ++p) {
    for (int q : B.probs[p].preds) B.pred.push_back(q);
    B.pred_off[p + 1] = (int)B.pred.size();
  }
  if (B.pred.empty()) B.pred.push_back(0);  // never read; keeps the device array non-empty
  return MSB_OK;
}

// Classes from the problems' (nm, nch) and the chosen tile per (nm, nch).
void make_classes(BatchImpl& B, const std::map<std::pair<int, int>, bool>& tile24) {
  std::map<int, int> kind_to_cls;
  B.classes.clear();
  std::map<int, double> work;
  for (auto& p : B.probs) {
    auto it = tile24.find({p.d.nm, p.nch});
    const bool t24 = it != tile24.end() && it->second;
    p.kind = batch_kind(p.d.nm, p.nch, t24);
    p.tx = t24 ? 2 : 4;
    p.ty = t24 ? 4 : 2;
    work[p.kind] += p.work;
  }
  // classes in increasing kind order: the kernel visits the kinds in that order
  for (auto& k : work) {
    ClassInfo c;
    c.kind = k.first;
    c.work = k.second;
    kind_to_cls[c.kind] = (int)B.classes.size();
    B.classes.push_back(c);
  }
  for (auto& p : B.probs) {
    p.cls = kind_to_cls[p.kind];
    ClassInfo& c = B.classes[p.cls];
    c.nm = p.d.nm;
    c.nch = p.nch;
    c.tx = p.tx;
    c.ty = p.ty;
  }
}

// Plans every problem, then the arena (scratch_bytes, or all the problems'
// scratch capped at `cap`) and the task table.
int plan_batch(BatchImpl& B, const msb_problem* probs, int n, const std::map<std::pair<int, int>, bool>& tile24,
               size_t scratch_bytes, size_t cap) {
  // one entry per 32-angle pass of every problem
  B.probs.clear();
  B.nuser = n;
  std::vector<int> first_entry(n);
  for (int i = 0; i < n; ++i) {
    const int npass = (probs[i].na + 31) / 32;
    first_entry[i] = (int)B.probs.size();
    auto it = tile24.find({probs[i].nm, 1});
    const bool t24 = it != tile24.end() && it->second;
    for (int c = 0; c < npass; ++c) {
      ProbPlan e;
      e.d = probs[i];
      e.user = i;
      e.pass = c;
      e.npass = npass;
      e.a0 = 32 * c;
      e.nac = std::min(32, probs[i].na - 32 * c);
      e.prev = c > 0 ? (int)B.probs.size() - 1 : -1;
      e.nch = 1;
      e.tx = t24 ? 2 : 4;
      e.ty = t24 ? 4 : 2;
      if (c > 0) B.probs.back().next = (int)B.probs.size();
      B.probs.push_back(e);
    }
  }
  // the problems' schedules are independent: build them on the host's cores
  // (a problem's passes share its schedule)
  std::vector<int> prc(n, MSB_OK);
  {
    const int nthr = std::max(1, std::min<int>(n, (int)std::thread::hardware_concurrency()));
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < nthr; ++t)
      pool.emplace_back([&]() {
        for (int i = next++; i < n; i = next++) prc[i] = plan_problem(B.probs[first_entry[i]], B.nsm);
      });
    for (auto& th : pool) th.join();
  }
  for (int i = 0; i < n; ++i)
    if (prc[i]) return plan_problem(B.probs[first_entry[i]], B.nsm);  // again on this thread: its error message
  for (auto& e : B.probs)
    if (e.pass > 0) {
      const ProbPlan& f = B.probs[e.prev];
      e.ngp = f.ngp;
      e.sched = f.sched;
      for (int k = 0; k < 3; ++k) e.face_bytes[k] = f.face_bytes[k];
      e.scratch = f.scratch;
      e.work = f.work;
    }
  make_classes(B, tile24);
  if ((int)B.classes.size() > kMaxBatchClasses) return set_error(MSB_ERR_ARG, "batch: too many classes");
  size_t need = 0;
  for (auto& p : B.probs)
    if (p.pass == 0) need += p.scratch;
  B.arena_bytes = scratch_bytes ? scratch_bytes : std::min(need, cap);
  return simulate_and_order(B);
}

template <class T>
int upload(T** dst, const std::vector<T>& v, const char* what) {
  int rc = cuda_check(cudaMalloc(dst, std::max<size_t>(1, v.size()) * sizeof(T)), what);
  if (rc) return rc;
  if (v.empty()) return MSB_OK;
  return cuda_check(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), what);
}

int setup_kernel(int* nsm) {
  static bool done = false;
  static int sm = 0;
  int rc, dev = 0;
  if ((rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice"))) return rc;
  if ((rc = cuda_check(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev), "SM count"))) return rc;
  constexpr size_t smem = fp64_batch_smem<kBatchStages>();
  static_assert(smem <= 227 * 1024 - 1024, "shared memory budget of the batched kernel");
  if (!done) {
    if ((rc = cuda_check(cudaFuncSetAttribute(sweep_fp64_batch_kernel<kBatchStages>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                         "cudaFuncSetAttribute (batch)")))
      return rc;
    int occ = 0;
    if ((rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, sweep_fp64_batch_kernel<kBatchStages>,
                                                                       384, smem),
                         "occupancy (batch)")))
      return rc;
    if (occ < 1) return set_error(MSB_ERR_UNSUPPORTED, "batched sweep kernel does not fit on an SM");
    done = true;
  }
  *nsm = sm;
  return MSB_OK;
}

// Device buffers of a planned batch.
int upload_batch(BatchImpl& B) {
  int rc;
  B.free_device();
  if ((rc = cuda_check(cudaMalloc(&B.d_arena, std::max<size_t>(B.arena_bytes, kAlign)), "cudaMalloc batch arena")))
    return rc;
  std::vector<Fp64Prob> pv(B.probs.size());
  for (size_t i = 0; i < B.probs.size(); ++i) {
    const ProbPlan& P = B.probs[i];
    Fp64Prob& q = pv[i];
    q.vi = P.d.vi;
    q.vo = P.d.vo;
    // the pass's angles of the caller's matrices, read in place
    q.afm = P.d.a_from_m ? P.d.a_from_m + P.a0 : nullptr;
    q.mfa = P.d.m_from_a ? P.d.m_from_a + (size_t)P.a0 * P.d.nm : nullptr;
    q.a_stride = P.d.na;
    unsigned char* base = static_cast<unsigned char*>(B.d_arena) + P.offset;
    q.fxy = reinterpret_cast<double*>(base);
    q.fxz = reinterpret_cast<double*>(base + P.face_bytes[0]);
    q.fyz = reinterpret_cast<double*>(base + P.face_bytes[0] + P.face_bytes[1]);
    q.nx = P.d.ncell_x;
    q.ny = P.d.ncell_y;
    q.nz = P.d.ncell_z;
    q.ne = P.d.ne;
    q.na = P.nac;
    q.ngp = P.ngp;
    q.ia_base = P.a0;
    q.vo_add = P.pass > 0 ? 1 : 0;
    q.ie_base = 0;
  }
  if ((rc = upload(&B.d_tasks, B.rec, "batch tasks"))) return rc;
  if ((rc = upload(&B.d_task_prob, B.task_prob, "batch task problems"))) return rc;
  if ((rc = upload(&B.d_probs, pv, "batch problems"))) return rc;
  if ((rc = upload(&B.d_pred_off, B.pred_off, "batch predecessors"))) return rc;
  if ((rc = upload(&B.d_pred, B.pred, "batch predecessors"))) return rc;
  if ((rc = upload(&B.d_prob_ntask, B.prob_ntask, "batch task counts"))) return rc;
  B.sync_ints = SY_PROGRESS + (size_t)B.ntask + B.probs.size();
  if ((rc = cuda_check(cudaMalloc(&B.d_sync, B.sync_ints * sizeof(int)), "cudaMalloc batch sync"))) return rc;
  if ((rc = cuda_check(cudaMalloc(&B.d_ptime, (B.probs.size() + 1) * sizeof(long long)), "cudaMalloc batch times")))
    return rc;
  if ((rc = cuda_check(cudaMallocHost(&B.h_status, 8 * sizeof(int)), "cudaMallocHost batch status"))) return rc;
  B.device = true;
  return MSB_OK;
}

Fp64Batch launch_params(const BatchImpl& B, int dir) {
  Fp64Batch P;
  memset(&P, 0, sizeof P);
  P.tasks = B.d_tasks;
  P.task_prob = B.d_task_prob;
  P.probs = B.d_probs;
  P.pred_off = B.d_pred_off;
  P.pred = B.d_pred;
  P.prob_ntask = B.d_prob_ntask;
  P.pdone = B.d_sync + SY_PROGRESS + B.ntask;
  P.ptime = B.d_ptime;
  P.nclass = (int)B.classes.size();
  for (int c = 0; c < P.nclass; ++c) {
    P.cls_base[c] = B.classes[c].base;
    P.cls_ntask[c] = B.classes[c].ntask;
    P.cls_kind[c] = B.classes[c].kind;
  }
  P.nprob = (int)B.probs.size();
  P.dir = dir;
  P.sy.sync = B.d_sync;
  P.sy.timeout_ns = B.timeout_ns;
  return P;
}

// One batched sweep on `st` (asynchronous).
int enqueue_sweep(BatchImpl& B, int dir, cudaStream_t st) {
  int rc;
  if ((rc = cuda_check(cudaMemsetAsync(B.d_sync, 0, B.sync_ints * sizeof(int), st), "reset batch sync"))) return rc;
  const Fp64Batch P = launch_params(B, dir);
  const int grid = (int)std::min<long long>(B.ntask, (long long)B.nsm);
  sweep_fp64_batch_kernel<kBatchStages><<<grid, 384, fp64_batch_smem<kBatchStages>(), st>>>(P);
  return cuda_check(cudaGetLastError(), "batched sweep launch");
}

int enqueue_status(BatchImpl& B, cudaStream_t st) {
  return cuda_check(cudaMemcpyAsync(B.h_status, B.d_sync, 4 * sizeof(int), cudaMemcpyDeviceToHost, st),
                    "batch status copy");
}

int sync_status(BatchImpl& B, cudaStream_t st) {
  int rc;
  if ((rc = cuda_check(cudaStreamSynchronize(st), "batched sweep"))) return rc;
  const int err = B.h_status[SY_ERROR];
  if (err == MSB_ERR_TIMEOUT)
    return set_error(MSB_ERR_TIMEOUT, "a device wait ran out of time (task %d); batched sweep aborted",
                     B.h_status[SY_ERRTASK]);
  if (err) return set_error(err, "device error %d in the batched sweep", err);
  return MSB_OK;
}

// Times both tile shapes on the median problem of each nm group (every
// entry sweeps one 32-angle chunk) and returns the faster shape per group.  The trial sweeps write that problem's
// vo array (the batch's own sweeps overwrite it later).
int autotune(const msb_problem* probs, int n, int nsm, size_t arena, std::map<std::pair<int, int>, bool>* tile24,
             double* tune_ms) {
  std::map<std::pair<int, int>, std::vector<int>> groups;
  for (int i = 0; i < n; ++i) groups[{probs[i].nm, 1}].push_back(i);
  cudaStream_t st = nullptr;
  int rc = cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "autotune stream");
  if (rc) return rc;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double total = 0.0;
  for (auto& g : groups) {
    std::vector<int>& v = g.second;
    auto cells = [&](int i) {
      const msb_problem& p = probs[i];
      return (double)p.ncell_x * p.ncell_y * p.ncell_z * p.ne * p.na;
    };
    std::sort(v.begin(), v.end(), [&](int a, int b) { return cells(a) < cells(b); });
    const int rep = v[v.size() / 2];
    double best = 1e30;
    bool best24 = false;
    for (int t24 = 0; t24 < 2 && !rc; ++t24) {
      BatchImpl T;
      T.nsm = nsm;
      std::map<std::pair<int, int>, bool> choice{{g.first, t24 != 0}};
      if ((rc = plan_batch(T, &probs[rep], 1, choice, 0, arena))) break;
      if ((rc = upload_batch(T))) break;
      float ms = 0.f, acc = 0.f;
      for (int it = 0; it < 3 && !rc; ++it) {
        cudaEventRecord(e0, st);
        rc = enqueue_sweep(T, 0, st);
        cudaEventRecord(e1, st);
        if (!rc) rc = enqueue_status(T, st);
        if (!rc) rc = sync_status(T, st);
        cudaEventElapsedTime(&ms, e0, e1);
        if (it > 0) acc += ms;
      }
      total += acc;
      if (!rc && acc < best) {
        best = acc;
        best24 = t24 != 0;
      }
    }
    (*tile24)[g.first] = best24;
    if (rc) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  if (tune_ms) *tune_ms = total;
  return rc;
}

}  // namespace
}  // namespace msb

using msb::BatchImpl;

struct msb_batch {
  BatchImpl impl;
  double tune_ms = 0.0;
  int tile24[3][2] = {{0, 0}, {0, 0}, {0, 0}};
};

static int batch_build(msb_batch** out, const msb_problem* problems, int nproblem, int precision,
                       size_t scratch_bytes, int autotune_flag, int nsm_plan) {
  if (!out || !problems || nproblem <= 0) return msb::set_error(MSB_ERR_ARG, "batch: no problems");
  *out = nullptr;
  if (precision != 0) return msb::set_error(MSB_ERR_UNSUPPORTED, "batch: precision %d (batches sweep in FP64)", precision);
  const bool device = nsm_plan <= 0;
  int rc;
  for (int i = 0; i < nproblem; ++i)
    if ((rc = msb::check_problem(problems[i], i, device))) return rc;
  std::unique_ptr<msb_batch> b(new (std::nothrow) msb_batch());
  if (!b) return msb::set_error(MSB_ERR_ARG, "out of host memory");
  BatchImpl& B = b->impl;
  if (device) {
    if ((rc = msb::setup_kernel(&B.nsm))) return rc;
  } else {
    B.nsm = nsm_plan;
  }
  // arena: the given size, or all the face scratch the problems would need
  // at once, capped at 80 % of the free device memory
  size_t cap = ~(size_t)0;
  if (device) {
    size_t fr = 0, tot = 0;
    if ((rc = msb::cuda_check(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo"))) return rc;
    cap = (size_t)(fr * 0.8);
  }
  std::map<std::pair<int, int>, bool> tile24;
  if (autotune_flag && device) {
    if ((rc = msb::autotune(problems, nproblem, B.nsm, scratch_bytes ? scratch_bytes : cap, &tile24, &b->tune_ms)))
      return rc;
  }
  for (auto& t : tile24) {
    const int ni = t.first.first == 4 ? 0 : t.first.first == 8 ? 1 : 2;
    b->tile24[ni][t.first.second - 1] = t.second ? 1 : 0;
  }
  if ((rc = msb::plan_batch(B, problems, nproblem, tile24, scratch_bytes, cap))) return rc;
  if (device && (rc = msb::upload_batch(B))) return rc;
  *out = b.release();
  return MSB_OK;
}

extern "C" int msb_batch_create(msb_batch** out, const msb_problem* problems, int nproblem, int precision,
                                size_t scratch_bytes, int autotune) {
  return batch_build(out, problems, nproblem, precision, scratch_bytes, autotune, 0);
}

extern "C" int msb_batch_plan(msb_batch** out, const msb_problem* problems, int nproblem, int nsm,
                              size_t scratch_bytes, int tile24_mask) {
  if (nsm <= 0) return msb::set_error(MSB_ERR_ARG, "batch plan: nsm must be positive");
  if (!out || !problems || nproblem <= 0) return msb::set_error(MSB_ERR_ARG, "batch: no problems");
  *out = nullptr;
  int rc;
  for (int i = 0; i < nproblem; ++i)
    if ((rc = msb::check_problem(problems[i], i, false))) return rc;
  std::unique_ptr<msb_batch> b(new (std::nothrow) msb_batch());
  if (!b) return msb::set_error(MSB_ERR_ARG, "out of host memory");
  BatchImpl& B = b->impl;
  B.nsm = nsm;
  // bit (nm index) of the mask selects the 2 x 4 tile
  std::map<std::pair<int, int>, bool> tile24;
  const int nms[3] = {4, 8, 16};
  for (int k = 0; k < 3; ++k) tile24[{nms[k], 1}] = ((tile24_mask >> k) & 1) != 0;
  if ((rc = msb::plan_batch(B, problems, nproblem, tile24, scratch_bytes, ~(size_t)0))) return rc;
  *out = b.release();
  return MSB_OK;
}

extern "C" void msb_batch_destroy(msb_batch* b) { delete b; }

extern "C" int msb_batch_sweep(msb_batch* b, int dir, void* stream) {
  if (!b || !b->impl.device) return msb::set_error(MSB_ERR_ARG, "batch: not created on a device");
  if (dir != 0 && dir != 1) return msb::set_error(MSB_ERR_ARG, "batch: dir must be 0 or 1");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = msb::enqueue_sweep(b->impl, dir, st);
  if (!rc) rc = msb::enqueue_status(b->impl, st);
  b->impl.launches = 1;
  return rc;
}

extern "C" int msb_batch_run(msb_batch* b, int niterations, void* stream) {
  if (!b || !b->impl.device) return msb::set_error(MSB_ERR_ARG, "batch: not created on a device");
  if (niterations < 0) return msb::set_error(MSB_ERR_ARG, "batch: negative iteration count");
  BatchImpl& B = b->impl;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc;
  if (niterations == 0) return MSB_OK;
  if (B.graph_iters != niterations) {
    if (B.graph) cudaGraphExecDestroy(B.graph);
    B.graph = nullptr;
    B.graph_iters = -1;
    cudaStream_t cap = nullptr;
    if ((rc = msb::cuda_check(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "capture stream"))) return rc;
    cudaGraph_t g = nullptr;
    rc = msb::cuda_check(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "begin capture");
    for (int it = 0; it < niterations && !rc; ++it) rc = msb::enqueue_sweep(B, it & 1, cap);
    if (!rc) rc = msb::enqueue_status(B, cap);
    const int rc2 = msb::cuda_check(cudaStreamEndCapture(cap, &g), "end capture");
    if (!rc) rc = rc2;
    if (!rc) rc = msb::cuda_check(cudaGraphInstantiate(&B.graph, g, 0), "graph instantiate");
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cap);
    if (rc) return rc;
    B.graph_iters = niterations;
  }
  B.launches = niterations;
  return msb::cuda_check(cudaGraphLaunch(B.graph, st), "graph launch");
}

extern "C" int msb_batch_sync(msb_batch* b, void* stream) {
  if (!b || !b->impl.device) return msb::set_error(MSB_ERR_ARG, "batch: not created on a device");
  return msb::sync_status(b->impl, static_cast<cudaStream_t>(stream));
}

extern "C" int msb_batch_problem_ms(const msb_batch* b, double* ms, int n) {
  if (!b || !b->impl.device || !ms) return msb::set_error(MSB_ERR_ARG, "batch: invalid argument");
  const BatchImpl& B = b->impl;
  const int np = (int)B.probs.size();
  if (n < B.nuser) return msb::set_error(MSB_ERR_ARG, "batch: output holds %d values, %d problems", n, B.nuser);
  std::vector<long long> t(np + 1);
  int rc = msb::cuda_check(cudaMemcpy(t.data(), B.d_ptime, (np + 1) * sizeof(long long), cudaMemcpyDeviceToHost),
                           "batch times");
  if (rc) return rc;
  for (int u = 0; u < B.nuser; ++u) ms[u] = 0.0;
  for (int p = 0; p < np; ++p)  // a problem completes with its last pass
    if (B.probs[p].next < 0) ms[B.probs[p].user] = (double)(t[p] - t[np]) * 1e-6;
  return MSB_OK;
}

extern "C" int msb_batch_info(const msb_batch* b, msb_batch_info_t* info) {
  if (!b || !info) return msb::set_error(MSB_ERR_ARG, "batch: invalid argument");
  const BatchImpl& B = b->impl;
  memset(info, 0, sizeof *info);
  info->nproblem = B.nuser;
  info->ntask = B.ntask;
  info->nclass = (int)B.classes.size();
  info->scratch_bytes = B.arena_bytes;
  size_t need = 0;
  for (auto& p : B.probs)
    if (p.pass == 0) need += p.scratch;
  info->scratch_needed_all = need;
  info->npred = B.pred_off.empty() ? 0 : B.pred_off.back();
  info->nsm = B.nsm;
  info->sim_makespan = B.sim_makespan;
  info->sim_busy = B.sim_busy;
  info->tune_ms = b->tune_ms;
  for (int c = 0; c < info->nclass && c < MSB_BATCH_MAX_CLASSES; ++c) {
    info->class_nm[c] = B.classes[c].nm;
    info->class_nch[c] = B.classes[c].nch;
    info->class_tx[c] = B.classes[c].tx;
    info->class_ty[c] = B.classes[c].ty;
    info->class_ntask[c] = B.classes[c].ntask;
  }
  return MSB_OK;
}

extern "C" long long msb_batch_tasks(const msb_batch* b, int* rec, int* prob, long long max_tasks) {
  if (!b) return msb::set_error(MSB_ERR_ARG, "batch: invalid argument");
  const BatchImpl& B = b->impl;
  const long long m = std::min(B.ntask, max_tasks);
  if (rec && m > 0) memcpy(rec, B.rec.data(), (size_t)m * MSB_TASK_INTS * sizeof(int));
  if (prob && m > 0) memcpy(prob, B.task_prob.data(), (size_t)m * sizeof(int));
  return B.ntask;
}

extern "C" int msb_batch_entries(const msb_batch* b, int* problem, int* angle0, int max_entries) {
  if (!b) return msb::set_error(MSB_ERR_ARG, "batch: invalid argument");
  const BatchImpl& B = b->impl;
  const int ne = (int)B.probs.size();
  for (int p = 0; p < ne && p < max_entries; ++p) {
    if (problem) problem[p] = B.probs[p].user;
    if (angle0) angle0[p] = B.probs[p].a0;
  }
  return ne;
}

extern "C" int msb_batch_scratch(const msb_batch* b, long long* offset, long long* bytes, int* pred_off, int* pred,
                                 int max_pred) {
  if (!b) return msb::set_error(MSB_ERR_ARG, "batch: invalid argument");
  const BatchImpl& B = b->impl;
  const int np = (int)B.probs.size();
  for (int p = 0; p < np; ++p) {
    if (offset) offset[p] = (long long)B.probs[p].offset;
    if (bytes) bytes[p] = (long long)B.probs[p].scratch;
    if (pred_off) pred_off[p] = B.pred_off[p];
  }
  if (pred_off) pred_off[np] = B.pred_off[np];
  const int npred = B.pred_off[np];
  if (pred) {
    if (max_pred < npred) return msb::set_error(MSB_ERR_ARG, "batch: %d predecessors, room for %d", npred, max_pred);
    for (int i = 0; i < npred; ++i) pred[i] = B.pred[i];
  }
  return npred;
}

extern "C" int msb_batch_set_spin_limit(msb_batch* b, long long limit) {
  if (!b) return msb::set_error(MSB_ERR_ARG, "batch: invalid argument");
  b->impl.timeout_ns = limit > 0 ? limit : msb::kBatchTimeoutNs;
  if (b->impl.graph) cudaGraphExecDestroy(b->impl.graph);
  b->impl.graph = nullptr;
  b->impl.graph_iters = -1;
  return MSB_OK;
}

extern "C" int msb_builtin_matrices(int nm, int na, double* a_from_m, double* m_from_a) {
  if (nm <= 0 || na <= 0 || !a_from_m || !m_from_a) return msb::set_error(MSB_ERR_ARG, "invalid argument");
  msb::build_am_matrices(nm, na, a_from_m, m_from_a);
  return MSB_OK;
}
