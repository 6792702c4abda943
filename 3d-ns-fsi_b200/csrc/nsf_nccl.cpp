// Run-time loader of NCCL (nsf_nccl.h).
#include "nsf_nccl.h"

#include <dlfcn.h>

#include <mutex>
#include <type_traits>

namespace nsf {

const NcclApi* nccl_api(std::string* why) {
  static NcclApi api{};
  static bool ok = false;
  static std::string err;
  static std::once_flag once;
  std::call_once(once, [] {
    // RTLD_NOLOAD first: a copy the process already holds (torch's) is the one to use
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL | RTLD_NOLOAD);
    if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
      const char* e = dlerror();
      err = std::string("libnccl.so.2 could not be loaded: ") + (e ? e : "unknown");
      return;
    }
    bool all = true;
    auto sym = [&](auto& fn, const char* name) {
      void* p = dlsym(h, name);
      if (!p) {
        all = false;
        err = std::string("libnccl.so.2 lacks ") + name;
      }
      fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(p);
    };
    sym(api.getUniqueId, "ncclGetUniqueId");
    sym(api.commInitRank, "ncclCommInitRank");
    sym(api.commDestroy, "ncclCommDestroy");
    sym(api.send, "ncclSend");
    sym(api.recv, "ncclRecv");
    sym(api.allGather, "ncclAllGather");
    sym(api.groupStart, "ncclGroupStart");
    sym(api.groupEnd, "ncclGroupEnd");
    sym(api.errorString, "ncclGetErrorString");
    ok = all;
  });
  if (!ok && why) *why = err;
  return ok ? &api : nullptr;
}

}  // namespace nsf
