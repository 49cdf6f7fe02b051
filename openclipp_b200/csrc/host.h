// Host-side objects behind the opaque ocip* handles.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <new>
#include <string>

#include "../../include/OpenCLIPP.h"
#include "internal.h"

namespace ocipb {

// Error carried to the C boundary, where it becomes the return code.
struct Error {
  int code;
  std::string msg;
};
[[noreturn]] void fail(int code, const std::string& msg);
void check_cuda(cudaError_t e, const char* what);
const char* error_name(int code);

// Counterpart of the reference's COpenCL (C++/OpenCL.cpp:48-69): one device
// and one in-order queue (a CUDA stream), plus scratch buffers the kernels
// reuse from call to call.
struct Context {
  enum ScratchSlot {
    kTemplateEnergy = 0,
    kPlanes = 1,
    kTensorAux = 2,
    kBackward = 3,
    kEnergyMap = 4,      // row energies of the tensor path
    kProductMap = 5,     // F64 product sums of templates tiled over launches
    kTemplateStats = 6,  // per-channel template energy (FP64)
    kIndexRecords = 7,   // per-warp best-match records of the fused reduction
    kIndexMap = 8,       // score map of ocipProximityIndx when no Dest is given
    kIndexScratch = 9,   // group results of the map-path index reduction
    kNumScratch = 10
  };
  int device = 0;
  int sm_count = 0;
  int cc_major = 0, cc_minor = 0;
  cudaStream_t stream = nullptr;
  // Device-to-host reads run here, after the event of the image's last
  // writer, so a read of one score map overlaps kernels queued after it.
  cudaStream_t copy_stream = nullptr;
  // Recorded on `stream` after work whose destinations are not tracked per
  // image (a replayed batch graph); every read also waits for it.
  cudaEvent_t untracked = nullptr;
  std::string name;
  int path = 1;       // ocipProximityPath; PLAIN by default (the drop-in)
  int last_path = 1;  // path that served the last proximity call
  int band_rows = 0;  // output rows per tensor work item; 0: chosen per launch
  void* scratch(int slot, size_t bytes);
  // The tensor-path kernels set a device flag (kTensorAux scratch) when a
  // bounded wait expires (the kernel then returns without finishing its
  // work). Called after the stream is synchronised: clears the flag and fails
  // with CL_OUT_OF_RESOURCES if it was set.
  void check_device_errors();
  ~Context();

 private:
  struct Scratch {
    void* ptr = nullptr;
    size_t bytes = 0;
  };
  Scratch scratch_[kNumScratch];
};

// Counterpart of the reference's Image (C++/Image.cpp:154-166) over a Buffer
// (C++/Buffer.cpp): a device buffer plus the caller's host buffer, which the
// image does not own.
struct Image {
  static constexpr uint32_t kMagic = 0x0C1F1A6Eu;
  uint32_t magic = kMagic;
  Context* ctx = nullptr;
  SImage desc{};
  void* host = nullptr;
  void* dev = nullptr;
  size_t pitch = 0;        // device row pitch, bytes (multiple of 128)
  bool in_device = false;  // Memory::m_isInDevice (C++/Buffer.cpp:30-43)
  cudaEvent_t written = nullptr;  // recorded on the context's stream after the last write
  // The device address was handed out (ocipGetImageDevicePtr): writes made
  // through it are not tracked, so a read waits for all of the context's
  // queued work.
  bool exposed = false;
  // Host buffer transfers: pageable memory is copied through the driver's
  // staging (about 7-13 GB/s here), page-locked memory at PCIe rate (about
  // 55 GB/s). A buffer that is already page-locked is detected at creation;
  // a pageable one is page-locked (cudaHostRegister, unregistered on
  // release) once the image has made kRegisterAfter transfers, which repays
  // the registration cost (about 0.6 ms per MB) for buffers a caller reuses.
  bool host_pinned = false;
  bool host_registered = false;
  int host_transfers = 0;
  static constexpr int kRegisterAfter = 4;
  size_t row_bytes() const {
    return (size_t)desc.Width * desc.Channels * type_bytes((int)desc.Type);
  }
};

// Program handle: the reference's MultiProgram subclasses that own temporary
// buffers (Integral: C++/programs/Integral.cpp:42-95).
struct Program {
  static constexpr uint32_t kMagic = 0x0C1F9E0Au;
  enum Kind { kIntegral = 1, kProximityFFT = 2, kProximityBatch = 3, kStatistics = 4 };
  uint32_t magic = kMagic;
  int kind = kIntegral;
  Context* ctx = nullptr;
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  struct TensorBatch* batch = nullptr;  // kProximityBatch
};

extern thread_local std::string g_last_error;
extern std::map<Context*, bool> g_contexts;
extern Context* g_current;

// Runs a C-ABI body, turning exceptions into the returned error code (the
// reference's H() macro, OpenCLIPP/OpenCLIPP.cpp:82).
#define OCIP_GUARD(...)                         \
  try {                                         \
    __VA_ARGS__;                                \
  } catch (const ocipb::Error& err_) {          \
    ocipb::g_last_error = err_.msg;             \
    return err_.code;                           \
  } catch (const std::bad_alloc&) {             \
    ocipb::g_last_error = "out of host memory"; \
    return CL_OUT_OF_HOST_MEMORY;               \
  }                                             \
  return CL_SUCCESS;

Context& current();
Image& image(ocipImage h);
void send(Image& img);
void send_if_needed(Image& img);
// The image's device buffer has been written by work just queued on the
// context's stream (a kernel or an upload): records its event.
void mark_written(Image& img);
// Work just queued on the context's stream wrote images that are not tracked
// one by one: every later read waits for it.
void mark_untracked_writes(Context& ctx);
DevImage dev_view(const Image& img);

}  // namespace ocipb
