// Test infrastructure, not product code.
//
// Link shim for the reference CPU build.  With GPU_ACCELERATE set to 0
// (db/db_impl.cc:44) the CPU DoCompactionWork is compiled, but db_impl.cc still
// compiles GPUWriteLevel0 and a few thread helpers (db/db_impl.cc:50-181) that
// name the LUDA GPU classes declared in cuda/cuda_common.h, and DBImpl holds a
// gpu::HostAndDeviceMemory member (db/db_impl.h:215).  Those GPU sources need
// moderngpu and cannot be built here, so this file defines the named symbols:
// the memory-holder constructor/destructor are no-ops (the member is never
// used on the CPU path), and every other entry point aborts if it is ever
// reached, which the CPU path never does.

#include <cstdio>
#include <cstdlib>

#include "cuda/cuda_common.h"

namespace leveldb {
namespace gpu {

[[noreturn]] static void Unreachable(const char* what) {
  std::fprintf(stderr, "reference GPU path reached in CPU oracle build: %s\n", what);
  std::abort();
}

HostAndDeviceMemory::HostAndDeviceMemory() {}
HostAndDeviceMemory::~HostAndDeviceMemory() {}
Stream::Stream() : s_(0) {}
Stream::~Stream() {}

void SSTDecode::DoDecode() { Unreachable("SSTDecode::DoDecode"); }
void SSTDecode::DoGPUDecode_1(WpSlice*, int) { Unreachable("SSTDecode::DoGPUDecode_1"); }
void SSTDecode::DoGPUDecode_2(WpSlice*, int) { Unreachable("SSTDecode::DoGPUDecode_2"); }
void SSTEncode::DoEncode_1(bool) { Unreachable("SSTEncode::DoEncode_1"); }
void SSTEncode::DoEncode_2(bool) { Unreachable("SSTEncode::DoEncode_2"); }
void SSTEncode::DoEncode_3() { Unreachable("SSTEncode::DoEncode_3"); }
void SSTEncode::DoEncode_4() { Unreachable("SSTEncode::DoEncode_4"); }
void cudaMemHtD(void*, void*, size_t) { Unreachable("cudaMemHtD"); }
void cudaMemDtH(void*, void*, size_t) { Unreachable("cudaMemDtH"); }

}  // namespace gpu
}  // namespace leveldb
