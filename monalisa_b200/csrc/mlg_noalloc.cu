// Adjoint gridding that allocates no memory.
//
// Some callers cannot allocate device memory at call time: a host program
// that reserved all of the GPU's memory for its own pool at start-up (a
// cudaMalloc would fail or take memory the pool counts on), or an embedding
// whose rules forbid allocation after initialisation.
// mlg_gridder_n2u_leight_noalloc gives them the on-the-fly Gaussian gridder
// of mlg_gridder_n2u_leight with device-resident inputs and outputs that the
// caller owns, and takes every scratch byte the tile-binned algorithm needs
// (per-tile counters, scan space, the (tile, sample) bins, partial tiles of
// split bins) from one file-scope device array of fixed size.  Nothing here
// calls cudaMalloc, cudaFree, cudaMallocAsync or an allocating library
// routine.  The tile-binned algorithm sizes its bins from counts it reads
// back to the host, so each call waits once on its stream (see the header).
#include <mutex>

#include "mlg_gridder.cuh"

namespace mlg {
namespace {

// Fixed capacity of the scratch array.  Every GPU that loads the library holds
// these bytes until the process exits.
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// In host code the array's name is only a host-side stand-in: the device
// address is fetched once per device (with that device current) and cached.
// The same set-up loads the gridding kernels, so that under CUDA's lazy
// module loading the array and the kernels take their device memory at this
// first call and never later.
int scratch_base(void** out) {
  static std::mutex mu;
  static void* base[128] = {};
  int dev = 0;
  MLG_CUDA(cudaGetDevice(&dev));
  MLG_CHECK(dev >= 0 && dev < 128, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(mu);
  if (!base[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return fail(MLG_ERR_CUDA, "cudaGetSymbolAddress of the gridding scratch failed: %s", cudaGetErrorString(e));
    MLG_TRY(leight_preload());
    base[dev] = p;
  }
  *out = base[dev];
  return MLG_OK;
}

}  // namespace
}  // namespace mlg

extern "C" int mlg_gridder_n2u_leight_noalloc(int imDim, const float* aReal, const float* aImag, const float* tx,
                                              const float* ty, const float* tz, const float* Dn, int nCh, int nPt,
                                              int Nx, int Ny, int Nz, int nWin, float kernelParam_1,
                                              float kernelParam_2, float* bReal, float* bImag, void* stream) {
  using namespace mlg;
  (void)kernelParam_2;  // unused by the reference kernel too
  MLG_CHECK(nPt >= 0, "nPt must be >= 0");
  MLG_CHECK(bReal && bImag, "NULL output");
  MLG_CHECK(nPt == 0 || (aReal && aImag && tx && Dn && (imDim < 2 || ty) && (imDim < 3 || tz)),
            "NULL input for nPt=%d", nPt);
  const int N[3] = {Nx, Ny, Nz};
  LeightGeom g;
  MLG_TRY(leight_geometry(imDim, nCh, N, nWin, kernelParam_1, g));
  const size_t counters = LeightWorkspace::align(LeightWorkspace::counters_bytes(g));
  MLG_CHECK(counters < kNoAllocScratchBytes,
            "grid of %lld cells needs %zu bytes of tile counters; the no-allocation scratch holds %zu bytes",
            g.Nu_tot, counters, kNoAllocScratchBytes);
  void* base = nullptr;
  MLG_TRY(scratch_base(&base));
  LeightInputs in;
  in.layout = Layout::kPointSplit;
  in.re = aReal;
  in.im = aImag;
  in.tx = tx;
  in.ty = imDim > 1 ? ty : nullptr;
  in.tz = imDim > 2 ? tz : nullptr;
  in.Dn = Dn;
  LeightOutput out;
  out.layout = Layout::kPointSplit;
  out.re = bReal;
  out.im = bImag;
  LeightWorkspace ws;
  ws.counters = base;
  ws.counters_cap = counters;
  ws.bins = static_cast<char*>(base) + counters;
  ws.bins_cap = kNoAllocScratchBytes - counters;
  ws.grow_bins = nullptr;  // a too-small scratch is an error, never an allocation
  return leight_run(g, in, nPt, out, ws, (cudaStream_t)stream);
}
