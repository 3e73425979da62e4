// sph-to-grid without any device-memory allocation.
//
// Some callers cannot call cudaMalloc: a simulation code that maps its particles in situ, between time
// steps, after handing all device memory to its own pool allocator (or that runs with a hard memory
// budget per rank), and latency-sensitive callers that cannot afford the implicit device-wide
// synchronisation a cudaMalloc or cudaFree can cause.  For them, kiwi_sph_to_grid_device_noalloc runs the
// same pipeline as kiwi_sph_to_grid_device with every scratch buffer (binning counts, bounding boxes,
// tile lists, sort buffers, counters) carved from one fixed, file-scope device array of
// KIWI_NOALLOC_SCRATCH_BYTES, which every GPU that loads the library holds until the process exits.
// The caller still provides the particle arrays and the output arrays, in device memory.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/kiwi_b200.h"
#include "engine.hpp"

namespace {

constexpr size_t kScratchBytes = (size_t)KIWI_NOALLOC_SCRATCH_BYTES;

// The scratch area.  In host code this name is only a host-side stand-in for the device symbol; its
// device address comes from cudaGetSymbolAddress at set-up, separately for every device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;

struct DeviceState {
    std::mutex setup_mutex;  // first calls from several host threads set the device up once
    bool ready = false;
    KiwiCtx ctx;  // stream set per call; scratch slots carved from the device's scratch area
};

DeviceState g_state[kMaxDevices];

void put_err(char* err, size_t err_len, const char* msg) {
    if (err && err_len > 0) {
        std::snprintf(err, err_len, "%s", msg);
    }
}

// Set-up for the current device, once: the device address of the scratch area, the kernel tables in
// constant memory and two timing events.  Must run before any stream capture on that device.
// A set-up that failed leaves nothing behind that a later attempt would duplicate.
int setup(int dev, char* err, size_t err_len) {
    DeviceState& s = g_state[dev];
    std::lock_guard<std::mutex> lock(s.setup_mutex);
    if (s.ready) return KIWI_OK;
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || ptr == nullptr) {
        char buf[256];
        std::snprintf(buf, sizeof buf, "cudaGetSymbolAddress of the scratch area failed on device %d: %s", dev,
                      cudaGetErrorString(e));
        put_err(err, err_len, buf);
        cudaGetLastError();
        return KIWI_ERR_CUDA;
    }
    s.ctx.device = dev;
    s.ctx.arena = static_cast<unsigned char*>(ptr);
    s.ctx.arena_bytes = kScratchBytes;
    for (int i = 0; i < 2; ++i) {
        if (s.ctx.ev[i] == nullptr && cudaEventCreate(&s.ctx.ev[i]) != cudaSuccess) {
            s.ctx.ev[i] = nullptr;
            put_err(err, err_len, "cudaEventCreate failed during set-up");
            cudaGetLastError();
            return KIWI_ERR_CUDA;
        }
    }
    if (kiwi_b200::fp64_init_tables(&s.ctx) != KIWI_OK) {
        put_err(err, err_len, s.ctx.err.c_str());
        return KIWI_ERR_CUDA;
    }
    s.ready = true;
    return KIWI_OK;
}

}  // namespace

extern "C" int kiwi_sph_to_grid_device_noalloc(void* stream, const KiwiParticles* particles,
                                               const KiwiCartGrid* grid, const KiwiKernelSel* kernel,
                                               int precision, double* density, double* vx, double* vy, double* vz,
                                               double* raw4, KiwiStats* stats, char* err, size_t err_len) {
    using namespace kiwi_b200;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        put_err(err, err_len, "no current CUDA device");
        return KIWI_ERR_NODEV;
    }
    int rc = setup(dev, err, err_len);
    if (rc != KIWI_OK) return rc;
    KiwiCtx* ctx = &g_state[dev].ctx;
    ctx->stream = static_cast<cudaStream_t>(stream);
    // every call carves its buffers afresh from the start of the scratch area
    ctx->arena_used = 0;
    for (int i = 0; i < KiwiCtx::kSlots; ++i) {
        ctx->slot_ptr[i] = nullptr;
        ctx->slot_bytes[i] = 0;
    }
    ctx->err.clear();
    rc = KIWI_OK;
    KernelChoice kc;
    CartGeom g;
    if (!particles_ok(ctx, particles, &rc)) {
    } else if ((rc = resolve_kernel(ctx, kernel, &kc)) != KIWI_OK) {
    } else if ((rc = make_geom(ctx, grid, kc.support_in_h, &g)) != KIWI_OK) {
    } else {
        DevParticles P{particles->n, particles->x, particles->y, particles->z, particles->vx,
                       particles->vy, particles->vz, particles->m, particles->h};
        CartOutputs out{density, vx, vy, vz, raw4, nullptr};
        rc = sph_to_grid_dev(ctx, P, g, kc, precision, out, stats);
    }
    if (rc != KIWI_OK) {
        put_err(err, err_len, ctx->err.c_str());
        // a failed call may have queued kernels that still write the shared array: let them finish, so
        // that the caller may reuse its buffers or call again on another stream at once
        cudaStreamSynchronize(ctx->stream);
        cudaGetLastError();
    }
    ctx->stream = nullptr;
    return rc;
}
