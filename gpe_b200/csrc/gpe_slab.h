// z-slab decomposition of one solve (the reference's MPI layout of
// src/variables.f90:203-375 with the y split dropped): slab r owns planes
// [k0, k0 + nzl) of the global grid and exchanges R boundary planes with
// its neighbours after every stage.  Two transports:
//   * NCCL (one process per GPU): ncclSend/ncclRecv of contiguous plane
//     blocks on the solve's stream; reductions by ncclAllReduce.  NCCL is
//     loaded at run time (dlopen), so single-GPU users never need it.
//   * an in-process hub: the slabs of one process, each driven by its own
//     host thread, on one device and one shared stream; exchanges are
//     device-to-device copies after a host barrier, reductions are summed
//     on the host in rank order.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <condition_variable>
#include <mutex>
#include <string>
#include <vector>

struct gpe_handle;

namespace gpe {

// Split nz planes over n ranks: the first nz % n ranks get one plane more.
void slab_partition(int nz, int n, int rank, int* k0, int* nzl);

// ---- NCCL, resolved at run time ------------------------------------------
// Opaque NCCL objects are carried as void* / 128-byte ids; the typed calls
// live in gpe_slab.cpp.
bool nccl_available(std::string& why);
int nccl_unique_id(void* id128, std::string& why);
int nccl_comm_init(void** comm, int nranks, const void* id128, int rank, std::string& why);
void nccl_comm_destroy(void* comm);
// one exchange round on stream st: every (send, recv) pair is posted inside
// one NCCL group.  peer < 0 skips the transfer.
struct NcclXfer {
  int peer;
  const void* send;
  void* recv;
  size_t bytes;
};
int nccl_exchange(void* comm, const NcclXfer* xs, int n, cudaStream_t st, std::string& why);
// dres[0..5]: sum slots 0,1,3,4 and max slots 2,5 over the ranks, in place
int nccl_reduce_results(void* comm, double* dres, cudaStream_t st, std::string& why);

// ---- in-process hub -------------------------------------------------------
struct SlabHub {
  int n = 0;
  int dev = 0;
  cudaStream_t st = nullptr;
  std::vector<gpe_handle*> slabs;
  std::vector<std::array<double, 6>> vals;
  std::mutex mu;
  std::condition_variable cv;
  int arrived = 0;
  long long gen = 0;
  bool broken = false;
  double timeout_s = 120.0;  // a barrier wait longer than this breaks the hub
  // waits for all n threads; false on timeout (the hub is then broken and
  // every later wait fails at once, so no thread is left behind)
  bool barrier(double timeout_s);
};

}  // namespace gpe
