// node_comm.cpp -- a process group on one node, for programs that drive the
// library through the reference's own C API (its sweep and tester drivers)
// with no transport of their own.
//
// The reference runs its decomposed sweep over MPI (env_mpi.c:100-480).  Here
// the processes of one node form the group: a launcher starts them with
// MSB_NPROC / MSB_PROC / MSB_GROUP in the environment, Env_initialize attaches
// each to a shared-memory segment named after the group and selects GPU
// proc % (GPUs visible).  The collectives (barrier, sum, allgather) run in
// that segment; the face messages go device to device: every receiving
// process publishes a CUDA IPC handle of its receive buffer, and the sender
// copies its send buffer straight into the peer's buffer (NVLink between
// GPUs, a device copy when both share one).  Waits are bounded (600 s); a
// process that stops answering makes the others fail with an error instead of
// hanging.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

#include <atomic>
#include <cstdlib>
#include <cstring>
#include <string>

#include "internal.h"

namespace msb {
namespace {

constexpr int kMaxProcs = 256;
constexpr long long kWaitNs = 600LL * 1000000000LL;

struct NodeSlot {
  cudaIpcMemHandle_t handle;
  unsigned long long offset;  // of the buffer inside the exported allocation
};

// One barrier: arrivals at the current one, and how many completed.
struct alignas(64) NodeBarrier {
  std::atomic<int> count;
  std::atomic<int> gen;
};

// The segment; zero-filled by ftruncate, so every counter starts at 0.  The
// collectives of the processes 0 .. n-1 use barrier n: a process that is
// idle in one run of the driver (the grid leaves it out) and goes on to the
// next run never mixes with the processes still in the first (the
// reference gives each run its own communicator, env_mpi.c:128-135).
struct NodeShared {
  NodeBarrier bar[kMaxProcs + 1];
  std::atomic<int> attached;  // processes that mapped the segment
  double dval[kMaxProcs];
  int ival[kMaxProcs];
  int dev_key[kMaxProcs];               // the GPU of each process (PCI location)
  NodeSlot slot[kMaxProcs][4];          // receive buffers: x lower / higher, y lower / higher
};
static_assert(std::atomic<int>::is_always_lock_free, "process-shared atomics");

struct Mapping {
  cudaIpcMemHandle_t handle;
  char* base = nullptr;
};

struct NodeState {
  NodeShared* sh = nullptr;
  int proc = 0, nproc = 1;
  cudaStream_t stream = nullptr;
  Mapping map[kMaxProcs][4];  // peers' receive buffers opened here
};

NodeState g_node;
msb_comm g_comm;

long long now_ns() {
  timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec * 1000000000LL + t.tv_nsec;
}

int node_barrier(void*, int nactive) {
  if (nactive < 1 || nactive > g_node.nproc || g_node.proc >= nactive)
    return set_error(MSB_ERR_ARG, "process group: barrier of %d processes from process %d", nactive, g_node.proc);
  NodeBarrier* s = &g_node.sh->bar[nactive];
  const int gen = s->gen.load(std::memory_order_acquire);
  if (s->count.fetch_add(1, std::memory_order_acq_rel) == nactive - 1) {
    // the last arrival resets the count before it releases the others
    s->count.store(0, std::memory_order_relaxed);
    s->gen.fetch_add(1, std::memory_order_acq_rel);
    return 0;
  }
  const long long t0 = now_ns();
  for (unsigned spin = 0; s->gen.load(std::memory_order_acquire) == gen; ++spin) {
    if (spin > 256) {
      timespec ts{0, 20000};
      nanosleep(&ts, nullptr);
    }
    if (now_ns() - t0 > kWaitNs)
      return set_error(MSB_ERR_TIMEOUT, "process group: no barrier partner for 600 s (process %d)", g_node.proc);
  }
  return 0;
}

int node_sum(void*, int nactive, double* v) {
  g_node.sh->dval[g_node.proc] = *v;
  if (node_barrier(nullptr, nactive)) return -1;
  double s = 0.0;
  for (int q = 0; q < nactive; ++q) s += g_node.sh->dval[q];  // the same order everywhere
  if (node_barrier(nullptr, nactive)) return -1;
  *v = s;
  return 0;
}

int node_allgather(void*, int nactive, int value, int* values) {
  g_node.sh->ival[g_node.proc] = value;
  if (node_barrier(nullptr, nactive)) return -1;
  for (int q = 0; q < nactive; ++q) values[q] = g_node.sh->ival[q];
  return node_barrier(nullptr, nactive) ? -1 : 0;
}

// Start of the allocation that holds `p` (an IPC handle names a whole
// allocation).
int allocation_base(const void* p, char** base) {
  static PFN_cuMemGetAddressRange_v3020 fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return set_error(MSB_ERR_CUDA, "cuMemGetAddressRange is not available from the driver");
    fn = reinterpret_cast<PFN_cuMemGetAddressRange_v3020>(f);
  }
  CUdeviceptr b = 0;
  size_t n = 0;
  if (fn(&b, &n, (CUdeviceptr)(uintptr_t)p) != CUDA_SUCCESS)
    return set_error(MSB_ERR_CUDA, "cuMemGetAddressRange failed");
  *base = reinterpret_cast<char*>((uintptr_t)b);
  return MSB_OK;
}

int node_exchange(void*, int nactive, const msb_kba_msg* msgs, int nmsg) {
  NodeState& G = g_node;
  int rc = MSB_OK;
  // 1. publish the receive buffers of this step
  for (int i = 0; i < nmsg && !rc; ++i) {
    if (msgs[i].is_send) continue;
    char* base = nullptr;
    NodeSlot& sl = G.sh->slot[G.proc][2 * msgs[i].axis + msgs[i].side];
    rc = allocation_base(msgs[i].buf, &base);
    if (!rc) rc = cuda_check(cudaIpcGetMemHandle(&sl.handle, base), "cudaIpcGetMemHandle");
    if (!rc) sl.offset = (unsigned long long)(static_cast<char*>(msgs[i].buf) - base);
  }
  // every process is here: handles published, earlier receives unpacked
  if (node_barrier(nullptr, nactive)) return -1;
  // 2. copy every send into the peer's receive buffer
  for (int i = 0; i < nmsg && !rc; ++i) {
    const msb_kba_msg& m = msgs[i];
    if (!m.is_send) continue;
    const int s = 2 * m.axis + (1 - m.side);  // the peer receives from its other side
    const NodeSlot sl = G.sh->slot[m.peer][s];
    Mapping& mp = G.map[m.peer][s];
    if (!mp.base || memcmp(&mp.handle, &sl.handle, sizeof sl.handle) != 0) {
      if (mp.base) cudaIpcCloseMemHandle(mp.base);
      mp.base = nullptr;
      void* p = nullptr;
      rc = cuda_check(cudaIpcOpenMemHandle(&p, sl.handle, cudaIpcMemLazyEnablePeerAccess), "cudaIpcOpenMemHandle");
      if (rc) break;
      mp.base = static_cast<char*>(p);
      mp.handle = sl.handle;
    }
    rc = cuda_check(cudaMemcpyAsync(mp.base + sl.offset, m.buf, m.bytes, cudaMemcpyDeviceToDevice, G.stream),
                    "face message copy");
  }
  if (!rc) rc = cuda_check(cudaStreamSynchronize(G.stream), "face message copy");
  // every message has landed
  if (node_barrier(nullptr, nactive)) return -1;
  return rc ? -1 : 0;
}

int device_key() {
  int dev = 0, bus = 0, slot = 0, dom = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&bus, cudaDevAttrPciBusId, dev);
  cudaDeviceGetAttribute(&slot, cudaDevAttrPciDeviceId, dev);
  cudaDeviceGetAttribute(&dom, cudaDevAttrPciDomainId, dev);
  return (dom << 16) | (bus << 8) | slot;
}

}  // namespace

// Attaches this process to the group named in the environment, if any.
int node_attach(Env* env) {
  const char* sn = getenv("MSB_NPROC");
  const char* sp = getenv("MSB_PROC");
  const char* sg = getenv("MSB_GROUP");
  if (!sn || !sp || !sg) return MSB_OK;
  const int nproc = atoi(sn), proc = atoi(sp);
  if (nproc <= 1) return MSB_OK;
  if (nproc > kMaxProcs || proc < 0 || proc >= nproc)
    return set_error(MSB_ERR_ARG, "MSB_PROC %d of MSB_NPROC %d (at most %d processes)", proc, nproc, kMaxProcs);
  if (g_node.sh) return set_error(MSB_ERR_ARG, "this process is already in a group");
  // without a GPU the group still serves its collectives (host-side use)
  int ndev = 0, rc = MSB_OK;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess) {
    cudaGetLastError();
    ndev = 0;
  }
  if (ndev > 0 && (rc = cuda_check(cudaSetDevice(proc % ndev), "cudaSetDevice"))) return rc;
  const std::string name = std::string("/msb_") + sg;
  const int fd = shm_open(name.c_str(), O_CREAT | O_RDWR, 0600);
  if (fd < 0) return set_error(MSB_ERR_ARG, "shm_open %s failed", name.c_str());
  if (ftruncate(fd, sizeof(NodeShared)) != 0) {
    close(fd);
    return set_error(MSB_ERR_ARG, "ftruncate %s failed", name.c_str());
  }
  void* p = mmap(nullptr, sizeof(NodeShared), PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
  close(fd);
  if (p == MAP_FAILED) return set_error(MSB_ERR_ARG, "mmap %s failed", name.c_str());
  g_node.sh = static_cast<NodeShared*>(p);
  g_node.proc = proc;
  g_node.nproc = nproc;
  if (ndev > 0 && (rc = cuda_check(cudaStreamCreateWithFlags(&g_node.stream, cudaStreamNonBlocking), "stream")))
    return rc;
  g_node.sh->dev_key[proc] = ndev > 0 ? device_key() : -1 - proc;
  g_node.sh->attached.fetch_add(1, std::memory_order_acq_rel);
  if (node_barrier(nullptr, nproc)) return MSB_ERR_TIMEOUT;
  if (proc == 0) shm_unlink(name.c_str());  // everybody has it mapped
  int flags = 0;
  for (int q = 0; q < nproc; ++q)
    for (int r = q + 1; r < nproc; ++r)
      if (g_node.sh->dev_key[q] == g_node.sh->dev_key[r]) flags |= MSB_ENV_SHARED_GPU;
  g_comm.ctx = nullptr;
  g_comm.exchange = node_exchange;
  g_comm.sum_double = node_sum;
  g_comm.allgather_int = node_allgather;
  g_comm.barrier = node_barrier;
  env->flags_ = flags;
  return msb_env_set_comm(env, proc, nproc, &g_comm);
}

void node_detach(Env* env) {
  if (!g_node.sh || !env || env->comm_ != &g_comm) return;
  for (auto& row : g_node.map)
    for (auto& m : row)
      if (m.base) {
        cudaIpcCloseMemHandle(m.base);
        m.base = nullptr;
      }
  if (g_node.stream) cudaStreamDestroy(g_node.stream);
  munmap(g_node.sh, sizeof(NodeShared));
  g_node = NodeState();
  env->comm_ = nullptr;
}

}  // namespace msb
