// z-slab transports: NCCL loaded at run time, and the in-process hub.
#include "gpe_slab.h"

#include <dlfcn.h>
#include <nccl.h>

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <type_traits>

namespace gpe {

void slab_partition(int nz, int n, int rank, int* k0, int* nzl) {
  const int base = nz / n, extra = nz % n;
  *nzl = base + (rank < extra ? 1 : 0);
  *k0 = rank * base + (rank < extra ? rank : extra);
}

namespace {

struct Nccl {
  bool tried = false, ok = false;
  std::string why;
  ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  const char* (*GetErrorString)(ncclResult_t) = nullptr;
};

std::mutex g_nccl_mu;
Nccl g_nccl;

const Nccl& nccl(std::string& why) {
  std::lock_guard<std::mutex> lk(g_nccl_mu);
  if (!g_nccl.tried) {
    g_nccl.tried = true;
    // an NCCL already in the process (e.g. torch's) is reused
    void* lib = nullptr;
    if (const char* e = getenv("GPE_NCCL_LIB")) lib = dlopen(e, RTLD_NOW | RTLD_GLOBAL);
    if (!lib) lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!lib) lib = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    if (!lib) {
      g_nccl.why = "NCCL (libnccl.so.2) could not be loaded";
    } else {
      bool all = true;
      auto sym = [&](auto& fn, const char* name) {
        fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(lib, name));
        all = all && fn;
      };
      sym(g_nccl.GetUniqueId, "ncclGetUniqueId");
      sym(g_nccl.CommInitRank, "ncclCommInitRank");
      sym(g_nccl.CommDestroy, "ncclCommDestroy");
      sym(g_nccl.Send, "ncclSend");
      sym(g_nccl.Recv, "ncclRecv");
      sym(g_nccl.AllReduce, "ncclAllReduce");
      sym(g_nccl.GroupStart, "ncclGroupStart");
      sym(g_nccl.GroupEnd, "ncclGroupEnd");
      sym(g_nccl.GetErrorString, "ncclGetErrorString");
      g_nccl.ok = all;
      if (!all) g_nccl.why = "libnccl.so.2 lacks a required symbol";
    }
  }
  if (!g_nccl.ok) why = g_nccl.why;
  return g_nccl;
}

int fail_nccl(const Nccl& n, ncclResult_t r, const char* what, std::string& why) {
  why = std::string(what) + ": " + (n.GetErrorString ? n.GetErrorString(r) : "NCCL error");
  return -2;
}

}  // namespace

bool nccl_available(std::string& why) { return nccl(why).ok; }

int nccl_unique_id(void* id128, std::string& why) {
  const Nccl& n = nccl(why);
  if (!n.ok) return -2;
  static_assert(sizeof(ncclUniqueId) == 128, "ncclUniqueId is 128 bytes");
  ncclResult_t r = n.GetUniqueId(reinterpret_cast<ncclUniqueId*>(id128));
  return r == ncclSuccess ? 0 : fail_nccl(n, r, "ncclGetUniqueId", why);
}

int nccl_comm_init(void** comm, int nranks, const void* id128, int rank, std::string& why) {
  const Nccl& n = nccl(why);
  if (!n.ok) return -2;
  ncclUniqueId id;
  memcpy(&id, id128, sizeof(id));
  ncclComm_t c = nullptr;
  ncclResult_t r = n.CommInitRank(&c, nranks, id, rank);
  if (r != ncclSuccess) return fail_nccl(n, r, "ncclCommInitRank", why);
  *comm = c;
  return 0;
}

void nccl_comm_destroy(void* comm) {
  std::string why;
  const Nccl& n = nccl(why);
  if (n.ok && comm) n.CommDestroy(static_cast<ncclComm_t>(comm));
}

int nccl_exchange(void* comm, const NcclXfer* xs, int cnt, cudaStream_t st, std::string& why) {
  const Nccl& n = nccl(why);
  if (!n.ok) return -2;
  ncclComm_t c = static_cast<ncclComm_t>(comm);
  ncclResult_t r = n.GroupStart();
  if (r != ncclSuccess) return fail_nccl(n, r, "ncclGroupStart", why);
  for (int q = 0; q < cnt && r == ncclSuccess; ++q) {
    if (xs[q].peer < 0) continue;
    if (xs[q].send) r = n.Send(xs[q].send, xs[q].bytes, ncclChar, xs[q].peer, c, st);
    else r = n.Recv(xs[q].recv, xs[q].bytes, ncclChar, xs[q].peer, c, st);
  }
  const ncclResult_t r2 = n.GroupEnd();
  if (r != ncclSuccess) return fail_nccl(n, r, "ncclSend/ncclRecv", why);
  if (r2 != ncclSuccess) return fail_nccl(n, r2, "ncclGroupEnd", why);
  return 0;
}

int nccl_reduce_results(void* comm, double* dres, cudaStream_t st, std::string& why) {
  const Nccl& n = nccl(why);
  if (!n.ok) return -2;
  ncclComm_t c = static_cast<ncclComm_t>(comm);
  ncclResult_t r = n.GroupStart();
  if (r == ncclSuccess) r = n.AllReduce(dres, dres, 2, ncclDouble, ncclSum, c, st);
  if (r == ncclSuccess) r = n.AllReduce(dres + 3, dres + 3, 2, ncclDouble, ncclSum, c, st);
  if (r == ncclSuccess) r = n.AllReduce(dres + 2, dres + 2, 1, ncclDouble, ncclMax, c, st);
  if (r == ncclSuccess) r = n.AllReduce(dres + 5, dres + 5, 1, ncclDouble, ncclMax, c, st);
  const ncclResult_t r2 = n.GroupEnd();
  if (r != ncclSuccess) return fail_nccl(n, r, "ncclAllReduce", why);
  if (r2 != ncclSuccess) return fail_nccl(n, r2, "ncclGroupEnd", why);
  return 0;
}

bool SlabHub::barrier(double timeout_s) {
  std::unique_lock<std::mutex> lk(mu);
  if (broken) return false;
  const long long my = gen;
  if (++arrived == n) {
    arrived = 0;
    ++gen;
    cv.notify_all();
    return true;
  }
  const auto until = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
  while (gen == my && !broken) {
    if (cv.wait_until(lk, until) == std::cv_status::timeout && gen == my) {
      broken = true;
      cv.notify_all();
      return false;
    }
  }
  return !broken || gen != my;
}

}  // namespace gpe
