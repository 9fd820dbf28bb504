// convertAccumToDisplayNoAlloc: the display conversion with no allocation.
//
// convertAccumToDisplayCUDA stages the 8-bit image in a device buffer it
// allocates on first use (and reallocates when the size changes). Some callers
// cannot allocate device memory at the point where they want a frame: a
// renderer embedded in a host application whose device memory is owned by
// another allocator (a caching allocator that already holds the GPU's free
// memory, or a fixed memory budget), or an interactive loop that must not
// take the implicit device-wide synchronisation cudaMalloc/cudaFree bring.
// This variant stages the image in a fixed device array that is part of the
// library image instead.
//
// The staging array is a file-scope __device__ array of RB_NOALLOC_MAX_BYTES
// (8 MiB: width * height * channels up to 8,388,608, e.g. 2048 x 1024 RGBA or
// 1920 x 1080 RGB). Every GPU that loads the library holds it until the
// process exits. Its device address is looked up once per device (on the
// first call made with that device current) with cudaGetSymbolAddress; make
// that first call before any stream capture. All calls share the array and it
// keeps the previous call's bytes; the kernel writes every byte the call
// copies out, so nothing needs clearing. Calls that overlap on the GPU (from
// different host threads or streams) race on the array.
//
// The conversion kernel and the copy out run on the legacy default stream, as
// convertAccumToDisplayCUDA's callers expect: a caller that writes the
// accumulation from a non-blocking stream orders those writes before the call.
// The cached address does not survive cudaDeviceReset (the reset unloads the
// module that holds the array): a process that resets a device does not call
// this entry point on it again.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <string>

#include "rb_internal.hpp"

#define RB_NOALLOC_MAX_BYTES (8u << 20)
#define RB_NOALLOC_MAX_DEVICES 64

namespace rb {

static __device__ __align__(256) unsigned char g_display_scratch[RB_NOALLOC_MAX_BYTES];

static std::mutex g_noalloc_mu;
static unsigned char *g_scratch_addr[RB_NOALLOC_MAX_DEVICES] = {nullptr};

// Same per-pixel arithmetic as the display kernel of convertAccumToDisplayCUDA
// (gammaCorrectKernel, render_acc_kernel.cu:11-44).
// One thread per pixel on a 1-D grid, so any image that fits the array
// (a 1 x 2,796,202 RGB strip included) stays within the launch limits.
__global__ void k_gamma_static(const float4 *__restrict__ acc, unsigned char *__restrict__ out, int npix, int spp,
                               int ch, float gamma, const int *__restrict__ counts) {
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= npix) return;
  const float4 a = acc[pix];
  int n = counts ? abs(counts[pix]) : spp;
  if (n <= 0) n = 1;
  const float inv = 1.0f / (float)n, ig = 1.0f / gamma;
  const float r = fminf(powf(fmaxf(a.x * inv, 0.0f), ig), 0.999f);
  const float g = fminf(powf(fmaxf(a.y * inv, 0.0f), ig), 0.999f);
  const float b = fminf(powf(fmaxf(a.z * inv, 0.0f), ig), 0.999f);
  unsigned char *o = out + (size_t)pix * ch;
  o[0] = (unsigned char)(256.0f * r);
  o[1] = (unsigned char)(256.0f * g);
  o[2] = (unsigned char)(256.0f * b);
  if (ch == 4) o[3] = 255;
}

extern std::atomic<unsigned long long> g_launches;

}  // namespace rb

using namespace rb;

extern "C" int convertAccumToDisplayNoAlloc(void *d_accum_buffer, unsigned char *display_image, int width, int height,
                                            int channels, int num_samples, float gamma, void *d_pixel_sample_counts) {
  if (!d_accum_buffer || !display_image || width <= 0 || height <= 0 || num_samples <= 0 ||
      (channels != 3 && channels != 4)) {
    set_error("convertAccumToDisplayNoAlloc: invalid argument");
    return RB_ERR_INVALID_ARG;
  }
  const size_t bytes = (size_t)width * (size_t)height * (size_t)channels;
  if (bytes > RB_NOALLOC_MAX_BYTES) {
    set_error("convertAccumToDisplayNoAlloc: width * height * channels = " + std::to_string(bytes) +
              " bytes exceeds the fixed staging array of 8388608 bytes");
    return RB_ERR_CAPACITY;
  }
  int dev = 0;
  if (!cuda_ok(cudaGetDevice(&dev), "convertAccumToDisplayNoAlloc: cudaGetDevice")) return RB_ERR_CUDA;
  if (dev < 0 || dev >= RB_NOALLOC_MAX_DEVICES) {
    set_error("convertAccumToDisplayNoAlloc: device ordinal beyond 64");
    return RB_ERR_UNSUPPORTED;
  }
  unsigned char *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_scratch_addr[dev]) {
      void *p = nullptr;
      if (!cuda_ok(cudaGetSymbolAddress(&p, g_display_scratch), "convertAccumToDisplayNoAlloc: cudaGetSymbolAddress"))
        return RB_ERR_CUDA;
      g_scratch_addr[dev] = static_cast<unsigned char *>(p);
    }
    scratch = g_scratch_addr[dev];
  }
  // bytes <= 8 MiB and channels >= 3 bound the pixel count well inside int
  const int npix = width * height;
  k_gamma_static<<<(npix + 255) / 256, 256>>>(static_cast<const float4 *>(d_accum_buffer), scratch, npix, num_samples,
                                               channels, gamma, static_cast<const int *>(d_pixel_sample_counts));
  g_launches++;
  if (!cuda_ok(cudaGetLastError(), "convertAccumToDisplayNoAlloc: launch")) return RB_ERR_CUDA;
  if (!cuda_ok(cudaMemcpy(display_image, scratch, bytes, cudaMemcpyDeviceToHost),
               "convertAccumToDisplayNoAlloc: copy to host"))
    return RB_ERR_CUDA;
  return RB_OK;
}
