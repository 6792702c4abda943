// NCCL, loaded at run time (libnccl.so.2): the x-slab groups that span several processes move their planes
// with it. The library itself does not link NCCL, so single-process use needs none; a process that already
// loaded NCCL (e.g. through torch.distributed) shares that copy.
#ifndef NSF_NCCL_H
#define NSF_NCCL_H

#include <nccl.h>

#include <string>

namespace nsf {

struct NcclApi {
  ncclResult_t (*getUniqueId)(ncclUniqueId*);
  ncclResult_t (*commInitRank)(ncclComm_t*, int, ncclUniqueId, int);
  ncclResult_t (*commDestroy)(ncclComm_t);
  ncclResult_t (*send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
  ncclResult_t (*recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
  ncclResult_t (*allGather)(const void*, void*, size_t, ncclDataType_t, ncclComm_t, cudaStream_t);
  ncclResult_t (*groupStart)();
  ncclResult_t (*groupEnd)();
  const char* (*errorString)(ncclResult_t);
};

// The loaded API, or nullptr with *why set (library or symbol missing).
const NcclApi* nccl_api(std::string* why);

}  // namespace nsf
#endif
