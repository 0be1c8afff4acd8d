// hb_map2alm_f32_noalloc: the FP32 map2alm with its F(m, ring pair) scratch in a fixed
// file-scope device array instead of a caller-provided workspace.
//
// Who needs it: callers that must not allocate device memory per call and cannot hand over a
// workspace either -- a host runtime whose allocator is owned by someone else, or a plugin
// ABI with no slot for a workspace pointer.  The array is part of this library's device
// image: every GPU that loads the library holds HB_NOALLOC_SCRATCH_BYTES of it until the
// process exits.
//
// The computation is exactly hb_map2alm_f32's (ring analysis into F, then the Legendre
// analysis reading F); only where F lives differs.
#include <mutex>
#include <string>

#include "hb_internal.cuh"

namespace hb {
namespace {

constexpr size_t kScratchBytes = size_t(HB_NOALLOC_SCRATCH_BYTES);
constexpr int kMaxDevices = 64;

// The scratch array.  The host-side name is only a handle for the runtime; its device address
// comes from cudaGetSymbolAddress, once per device.
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
void *g_addr[kMaxDevices] = {};

// Device address of g_scratch on the current device; looked up on the first call made with
// that device current (this is where the runtime loads the module onto the device, if it has
// not done so yet) and cached afterwards.
int scratch_address(void **out) {
    int dev = -1;
    HB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(HB_ERR_UNSUPPORTED, "hb_map2alm_f32_noalloc: device ordinal " + std::to_string(dev) +
                                            " beyond the " + std::to_string(kMaxDevices) + " supported");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p)
            return fail(HB_ERR_CUDA, std::string("hb_map2alm_f32_noalloc: cudaGetSymbolAddress failed: ") +
                                         cudaGetErrorString(e));
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return HB_OK;
}

}  // namespace
}  // namespace hb

using namespace hb;

extern "C" int hb_map2alm_f32_noalloc(const hb_plan *p, int nmaps, const float *maps, const double *weights,
                                      float *alm, int flags, hb_stream_t stream) {
    if (!p || !p->g) return fail(HB_ERR_INVALID, "hb_map2alm_f32_noalloc: null plan");
    if (nmaps < 1 || nmaps > 65535) return fail(HB_ERR_INVALID, "hb_map2alm_f32_noalloc: nmaps must lie in [1, 65535]");
    const size_t need = hb_sht_workspace_size(p, 32, nmaps);
    if (need > kScratchBytes)
        return fail(HB_ERR_INVALID, "hb_map2alm_f32_noalloc: this call needs " + std::to_string(need) +
                                        " bytes of scratch (nmaps * (mmax+1) * npairs * 16), the static scratch "
                                        "holds " + std::to_string(kScratchBytes) +
                                        "; use hb_map2alm_f32 with a workspace or fewer maps per call");
    void *scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    return hb_map2alm_f32(p, nmaps, maps, weights, alm, scratch, kScratchBytes, flags, stream);
}
