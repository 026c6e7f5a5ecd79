// Out-of-core diffusion: volumes held in host memory (or files) that do not
// fit the device, processed as z-slabs with halos.
//
// The reference's out-of-core form (src/lib/cpp/gpu/diffusion.cc:947-1129)
// cuts the volume into 3-D blocks with a radius halo and exchanges halos
// through host memory on every repetition.  Here the volume is cut into
// z-slabs of S planes that span y and x, and a slab's value after k
// repetitions depends only on input planes within k x radius of it (one z pass
// per repetition).  Two plans follow from that:
//
//   * deep halos (the default): each slab is loaded once with H = R x radius
//     halo planes per cut side and all R repetitions run on the device; only
//     the slab's own planes are written back, and no exchange between slabs is
//     needed.  Repetition k runs only on the planes at least k x radius from a
//     cut side (the others can no longer reach the core), which brings the
//     computed planes per slab from R (S + 2H) to about R (S + H).
//   * exchange rounds, when R x radius halos leave no room for a useful slab:
//     the repetitions run in rounds of k, each slab carrying k x radius halo
//     planes; between rounds the slabs' FP32 fields go to a host copy of the
//     field (double-buffered, 8 bytes per voxel of pinned host memory) and the
//     next round starts from it.  FP32 results equal the in-memory form's.
//     Only where those 8 bytes per voxel fit half of the host's available
//     memory (MemAvailable; MAXIBONE_OOC_HOST_BUDGET overrides).
//
// A planner picks the slab depth (at most the caller's) and the plan from the
// free device memory and a cost estimate (voxel-repetitions computed, bytes
// crossing PCIe).  When the volume's plane is a multiple of 32 voxels the whole
// mask is uploaded once and kept bit-packed on the device (1/8 byte per voxel),
// so slabs need no mask uploads; from a pinned caller buffer the upload runs on
// its own stream in z order, and a slab's first kernel waits only for the
// chunks its planes lie in, so later planes cross PCIe while the first slabs
// compute.  The uint16 output of a slab is copied out on a
// second stream while the next slab's repetitions run (only its last
// repetition waits for that copy).  Pageable host buffers are staged through
// pinned memory by the host thread.
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <vector>
#include <functional>

#include "host_util.h"
#include "unrolled.h"

namespace maxi {

static bool is_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace maxi

using namespace maxi;

extern "C" int64_t maxi_diffusion_workspace_size(int64_t nz, int64_t ny, int64_t nx, int32_t field_type);

namespace maxi {

// Reads planes [z0, z0 + nzp) of the uint8 mask into `dst` (host memory).
using PlaneReader = std::function<int(int64_t z0, int64_t nzp, uint8_t *dst)>;
// Receives planes [z0, z0 + nzp) of the uint16 output from `src` (host memory).
using PlaneWriter = std::function<int(int64_t z0, int64_t nzp, const uint16_t *src)>;

// Slab plan: S core planes per slab, k repetitions per round (k == R: one
// round, deep halos), resident: the whole mask bit-packed on the device.
struct SlabPlan {
    int64_t S = 0, k = 0, E = 0;
    bool resident = false, shrinks = false;
    int64_t chunk_planes = 0;  // planes per upload chunk of a resident mask
    double cost = 0.0;         // estimated seconds
    bool host_limited = false;  // exchange rounds ruled out by the host memory they would pin
};

static int64_t field_size(int32_t ft) { return ft == MAXI_FIELD_F32 ? 4 : ft == MAXI_FIELD_F64 ? 8 : 2; }

// Largest output window over the slabs of a round of kr repetitions: the
// planes its last repetition computes, which the output buffers must hold.
// With shrinking windows that is the core and `radius` planes on each cut
// side, and down to the volume's edge where the halo reaches it; without
// shrinking, the whole extended slab.
static int64_t max_window(int64_t nz, int64_t S, int64_t radius, int64_t kr, bool shrinks) {
    const int64_t H = std::min(nz, kr * radius), n_slabs = ceil_div(nz, S);
    int64_t w = 0;
    for (int64_t s = 0; s < n_slabs; s++) {
        const int64_t z0 = s * S, z1 = std::min(nz, z0 + S);
        const int64_t e0 = std::max<int64_t>(0, z0 - H), e1 = std::min(nz, z1 + H);
        if (!shrinks) {
            w = std::max(w, e1 - e0);
            continue;
        }
        const int64_t ez = e1 - e0, j = std::max<int64_t>(0, kr - 1);
        const int64_t lo = std::min(ez - 1, (e0 > 0 ? radius : 0) * j);
        const int64_t hi = std::max(lo + 1, ez - (e1 < nz ? radius : 0) * j);
        w = std::max(w, hi - lo);
    }
    return w;
}

// Device bytes of one slab context: the workspace of an extended slab of E
// planes, its uint8 mask when the mask is not resident, and the output window
// of `win` planes (uint16; plus the FP32 field in exchange rounds).
static int64_t slab_bytes(int64_t E, int64_t win, int64_t plane, int32_t ft, bool resident, bool exchange) {
    const int64_t ws = maxi_diffusion_workspace_size(E, plane, 1, ft);
    return ws + (resident ? 0 : E * plane) + win * plane * (2 + (exchange ? 4 : 0)) + 4096;
}

// The window buffers of a plan: the largest window of its full rounds (k
// repetitions) and of its last round (the remainder).
static int64_t plan_window(int64_t nz, int64_t S, int64_t radius, int64_t reps, int64_t k, bool shrinks) {
    const int64_t last = reps > 0 ? reps - (ceil_div(reps, k) - 1) * k : 0;
    return std::max(max_window(nz, S, radius, k, shrinks), max_window(nz, S, radius, std::max<int64_t>(1, last), shrinks));
}

// Chooses the plan.  budget: device bytes available for the slab context.
static SlabPlan plan_slabs(int64_t nz, int64_t plane, int64_t radius, int64_t reps, int32_t ft, int64_t max_slab,
                           bool resident, bool allow_exchange, bool shrinks, int64_t budget) {
    SlabPlan best;
    best.cost = -1.0;
    const double vox_rate = 3e11, pcie = 4.5e10;  // rough voxel-repetitions/s and bytes/s for the estimate
    for (int64_t k = reps; k >= 1; k = (k == 1 ? 0 : std::max<int64_t>(1, (k + 1) / 2))) {
        const bool exchange = k < reps;
        if (exchange && !allow_exchange) break;
        const int64_t H = std::min(nz, k * radius);
        // Largest S with slab_bytes(S, min(nz, S + 2H)) <= budget (bisection; the
        // bytes grow with S).
        auto bytes_for = [&](int64_t S) {
            const int64_t n_slabs = ceil_div(nz, S), Sb = ceil_div(nz, n_slabs);  // balanced, as run
            return slab_bytes(std::min(nz, Sb + 2 * H), plan_window(nz, Sb, radius, reps, k, shrinks), plane, ft,
                              resident, exchange);
        };
        int64_t lo = 0, hi = std::min(nz, max_slab);
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) / 2;
            if (bytes_for(mid) <= budget) lo = mid;
            else hi = mid - 1;
        }
        // the balanced depth's bytes are not strictly monotonic: step down until it fits
        while (lo >= 1 && bytes_for(lo) > budget) lo--;
        if (lo >= 1) {
            const int64_t n_slabs = ceil_div(nz, lo), S = ceil_div(nz, n_slabs);  // balanced slabs
            const int64_t rounds = ceil_div(reps, k);
            // computed planes x repetitions: each cut side adds a halo that shrinks by radius per repetition
            double planes = 0.0;
            for (int64_t s = 0; s < n_slabs; s++) {
                const int64_t z0 = s * S, z1 = std::min(nz, z0 + S);
                const int cuts = (z0 > 0) + (z1 < nz);
                planes += (double) (z1 - z0) * reps + cuts * (double) radius * (double) (k * (k + 1) / 2) * rounds;
            }
            double bytes = (double) nz * plane * 3.0;                            // mask in, uint16 out
            if (exchange) bytes += (double) (rounds - 1) * nz * plane * 8.0 * 1.1;  // FP32 field out and back in
            const double cost = planes * plane / vox_rate + bytes / pcie;
            if (best.cost < 0.0 || cost < best.cost) {
                best.S = S;
                best.k = k;
                best.E = std::min(nz, S + 2 * H);
                best.resident = resident;
                best.cost = cost;
            }
        }
        if (k == 1) break;
    }
    return best;
}

// Device bytes the planner may use: the free bytes, or the value of the
// environment variable MAXIBONE_OOC_DEVICE_BUDGET when it is set (bytes; lets
// tests and callers that share the device plan for less).
static int64_t device_budget(size_t free_b) {
    const char *env = getenv("MAXIBONE_OOC_DEVICE_BUDGET");
    if (env && *env) {
        const long long v = atoll(env);
        if (v > 0) return std::min<int64_t>(v, (int64_t) free_b);
    }
    return (int64_t) free_b;
}

// Host bytes the exchange rounds may pin: half of the available memory
// (MemAvailable in /proc/meminfo), or the environment variable
// MAXIBONE_OOC_HOST_BUDGET (bytes) when it is set.
static int64_t host_budget() {
    const char *env = getenv("MAXIBONE_OOC_HOST_BUDGET");
    if (env && *env) {
        const long long v = atoll(env);
        if (v >= 0) return v;
    }
    long long kb = -1;
    if (FILE *f = fopen("/proc/meminfo", "r")) {
        char line[256];
        while (fgets(line, sizeof line, f))
            if (sscanf(line, "MemAvailable: %lld kB", &kb) == 1) break;
        fclose(f);
    }
    if (kb < 0) {
        const long pages = sysconf(_SC_AVPHYS_PAGES), page = sysconf(_SC_PAGESIZE);
        if (pages > 0 && page > 0) kb = (long long) pages * (page / 1024);
    }
    return kb > 0 ? (int64_t) kb * 1024 / 2 : 0;
}

// The whole plan for `free_b` device bytes and `host_b` pinnable host bytes:
// resident mask or not, whether the loop shrinks its window, then slab depth
// and repetitions per round.
static SlabPlan full_plan(int64_t nz, int64_t ny, int64_t nx, int64_t slab_z, int64_t kernel_size, int64_t repititions,
                          int32_t field_type, int32_t flags, int64_t free_b, int64_t host_b) {
    const int64_t plane = ny * nx, n = nz * plane;
    const int64_t radius = kernel_size / 2, R = std::max<int64_t>(1, repititions);
    const bool rebuild = (flags & MAXI_FLAG_MASK_FROM_FIELD) != 0;
    const int64_t reserve = std::min<int64_t>(free_b / 4, (int64_t(3) << 29) + free_b / 32);  // driver, descriptors
    int64_t budget = free_b - reserve;
    // Resident bit-packed mask: whole 32-bit words per plane, and small enough.
    const int64_t packed_bytes = round_up(ceil_div(n, 32) * 4, 256);
    // Upload chunks of about 1 GiB of mask (MAXIBONE_OOC_UPLOAD_CHUNK_PLANES planes when set).
    int64_t chunk_planes = std::max<int64_t>(1, std::min(nz, (int64_t(1) << 30) / plane));
    if (const char *env = getenv("MAXIBONE_OOC_UPLOAD_CHUNK_PLANES")) {
        const long long v = atoll(env);
        if (v > 0) chunk_planes = std::min<int64_t>(nz, v);
    }
    const bool resident = !rebuild && plane % 32 == 0 && repititions > 0 &&
                          packed_bytes + 2 * chunk_planes * plane < budget / 4;
    if (resident) budget -= packed_bytes + 2 * chunk_planes * plane;
    // Exchange rounds keep two FP32 fields on the host: not for the FP64 form,
    // and only where the host can pin them.
    const bool exchange_form = field_type != MAXI_FIELD_F64 && repititions > 1;
    const bool allow_exchange = exchange_form && 8 * n <= host_b;
    // The repetition loop shrinks its plane window towards the slab's core on
    // the unrolled passes (not the generic ones: FP64, reference rounding,
    // radius > 128) when planes are whole mask words.
    const bool shrinks = plane % 32 == 0 && field_type != MAXI_FIELD_F64 && radius <= 128 &&
                         !(flags & MAXI_FLAG_REFERENCE_ROUNDING);
    SlabPlan pl = plan_slabs(nz, plane, radius, R, field_type, slab_z > 0 ? slab_z : nz, resident, allow_exchange,
                             shrinks, budget);
    pl.resident = resident;
    pl.shrinks = shrinks;
    pl.chunk_planes = chunk_planes;
    pl.host_limited = exchange_form && !allow_exchange;
    return pl;
}

// The slab engine.  `direct_in` / `direct_out`: pinned caller buffers that the
// device copies can use without staging (may be NULL).  slab_z: the largest
// slab depth the caller allows (0: no limit).
static int run_slabs(int64_t nz, int64_t ny, int64_t nx, int64_t slab_z, const float *kernel, int64_t kernel_size,
                     int64_t repititions, int32_t field_type, int32_t flags, int verbose, const PlaneReader &read,
                     const PlaneWriter &write, const uint8_t *direct_in, uint16_t *direct_out) {
    const int64_t plane = ny * nx, n = nz * plane;
    const int64_t radius = kernel_size / 2;
    if (maxi_diffusion_workspace_size(1, ny, nx, field_type) < 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "unknown field_type %d", field_type);

    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const SlabPlan pl = full_plan(nz, ny, nx, slab_z, kernel_size, repititions, field_type, flags, device_budget(free_b),
                                  host_budget());
    const bool resident = pl.resident, shrinks = pl.shrinks;
    const int64_t packed_bytes = round_up(ceil_div(n, 32) * 4, 256), chunk_planes = pl.chunk_planes;
    if (pl.S < 1 && pl.host_limited)
        return set_error(MAXI_ERR_OUT_OF_MEMORY,
                         "%lld repetitions x radius %lld need halos of %lld planes per slab side, which leave no "
                         "slab that fits the %lld free bytes of the device, and rounds that exchange the field "
                         "through host memory need %lld bytes of pinned host memory (8 per voxel) where %lld may "
                         "be pinned (half of MemAvailable, or MAXIBONE_OOC_HOST_BUDGET)",
                         (long long) repititions, (long long) radius, (long long) std::min(nz, repititions * radius),
                         (long long) device_budget(free_b), (long long) (8 * n), (long long) host_budget());
    if (pl.S < 1)
        return set_error(MAXI_ERR_OUT_OF_MEMORY,
                         "no slab of whole %lld x %lld planes fits the %lld free bytes of the device (one plane with "
                         "a %lld-plane halo on each side needs %lld bytes); the volume's planes are too large for "
                         "this device",
                         (long long) ny, (long long) nx, (long long) device_budget(free_b), (long long) radius,
                         (long long) slab_bytes(std::min(nz, 1 + 2 * radius), std::min(nz, 1 + 2 * radius), plane,
                                                field_type, resident, true));
    const int64_t S = pl.S, k = std::min(pl.k, std::max<int64_t>(1, repititions)), E = pl.E;
    const bool exchange = k < repititions;
    const int64_t n_slabs = ceil_div(nz, S), rounds = repititions == 0 ? 1 : ceil_div(repititions, k);
    if (verbose >= 1)
        printf("Out-of-core diffusion: shape (%lld, %lld, %lld), %lld slabs of %lld planes, %lld round(s) of %lld "
               "repetitions with %lld-plane halos%s\n",
               (long long) nz, (long long) ny, (long long) nx, (long long) n_slabs, (long long) S, (long long) rounds,
               (long long) k, (long long) std::min(nz, k * radius), resident ? ", resident bit-packed mask" : "");

    // Device and host buffers.
    struct Buffers {
        cudaStream_t cs = nullptr, ds = nullptr;  // compute, download
        cudaStream_t us = nullptr;                // resident mask upload from a pinned caller buffer
        std::vector<cudaEvent_t> up;              // chunk c of that upload packed
        cudaEvent_t ready = nullptr, freed = nullptr;
        uint32_t *packed = nullptr;               // resident mask
        uint8_t *stage[2] = {nullptr, nullptr};   // resident mask upload chunks
        uint8_t *d_mask = nullptr;                // per-slab uint8 mask (not resident)
        void *ws = nullptr;
        uint16_t *d_out = nullptr;                // output window, S + 2 radius planes
        float *d_fwin = nullptr;                  // FP32 field window (exchange rounds)
        uint8_t *h_in = nullptr;                  // pinned staging (pageable input)
        uint16_t *h_out = nullptr;                // pinned staging (pageable output)
        float *h_field[2] = {nullptr, nullptr};   // host FP32 field, in / out of a round
        ~Buffers() {
            if (cs) cudaStreamSynchronize(cs);
            if (ds) cudaStreamSynchronize(ds);
            if (us) cudaStreamSynchronize(us);
            cudaFree(packed);
            cudaFree(stage[0]);
            cudaFree(stage[1]);
            cudaFree(d_mask);
            cudaFree(ws);
            cudaFree(d_out);
            cudaFree(d_fwin);
            cudaFreeHost(h_in);
            cudaFreeHost(h_out);
            cudaFreeHost(h_field[0]);
            cudaFreeHost(h_field[1]);
            if (ready) cudaEventDestroy(ready);
            if (freed) cudaEventDestroy(freed);
            for (cudaEvent_t ev : up) cudaEventDestroy(ev);
            if (cs) cudaStreamDestroy(cs);
            if (ds) cudaStreamDestroy(ds);
            if (us) cudaStreamDestroy(us);
        }
    } b;
    const int64_t ws_bytes = maxi_diffusion_workspace_size(E, ny, nx, field_type);
    const int64_t win = plan_window(nz, S, radius, repititions, k, shrinks);
    auto oom = [&](const char *what) {
        cudaGetLastError();
        return set_error(MAXI_ERR_OUT_OF_MEMORY, "could not allocate %s for slabs of %lld planes (%lld with halos)",
                         what, (long long) S, (long long) E);
    };
    if (cudaStreamCreateWithFlags(&b.cs, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b.ds, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b.ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b.freed, cudaEventDisableTiming) != cudaSuccess)
        return set_cuda_error(cudaGetLastError(), "out-of-core streams");
    const bool overlap_upload = resident && direct_in;
    if (overlap_upload) {
        if (cudaStreamCreateWithFlags(&b.us, cudaStreamNonBlocking) != cudaSuccess)
            return set_cuda_error(cudaGetLastError(), "out-of-core streams");
        for (int64_t z = 0; z < nz; z += chunk_planes) {
            b.up.push_back(nullptr);
            if (cudaEventCreateWithFlags(&b.up.back(), cudaEventDisableTiming) != cudaSuccess) {
                b.up.pop_back();
                return set_cuda_error(cudaGetLastError(), "out-of-core streams");
            }
        }
    }
    if (resident && (cudaMalloc(&b.packed, packed_bytes) != cudaSuccess ||
                     cudaMalloc(&b.stage[0], chunk_planes * plane) != cudaSuccess ||
                     cudaMalloc(&b.stage[1], chunk_planes * plane) != cudaSuccess))
        return oom("the resident bit-packed mask");
    if (cudaMalloc(&b.ws, ws_bytes) != cudaSuccess || cudaMalloc(&b.d_out, win * plane * 2) != cudaSuccess ||
        (!resident && cudaMalloc(&b.d_mask, E * plane) != cudaSuccess) ||
        (exchange && cudaMalloc(&b.d_fwin, win * plane * 4) != cudaSuccess))
        return oom("device slab buffers");
    if ((!direct_in && cudaMallocHost(&b.h_in, (resident ? chunk_planes : E) * plane) != cudaSuccess) ||
        (!direct_out && cudaMallocHost(&b.h_out, S * plane * 2) != cudaSuccess))
        return oom("pinned staging buffers");
    // Host copies of the field: written by device-to-host copies, read by the
    // next round's first kernel through their device mapping.
    float *d_field[2] = {nullptr, nullptr};
    if (exchange) {
        for (int i = 0; i < 2; i++)
            if (cudaHostAlloc(&b.h_field[i], n * 4, cudaHostAllocPortable | cudaHostAllocMapped) != cudaSuccess ||
                cudaHostGetDevicePointer(reinterpret_cast<void **>(&d_field[i]), b.h_field[i], 0) != cudaSuccess)
                return oom("the host copies of the field for exchange rounds (8 bytes per voxel of pinned memory)");
    }
    cudaError_t e;

    // Whole mask -> resident bit-packed words, chunk by chunk (the two staging
    // buffers alternate; the stream orders each refill after the previous
    // packing of that buffer).
    if (resident) {
        cudaStream_t ust = overlap_upload ? b.us : b.cs;
        for (int64_t z = 0, c = 0; z < nz; z += chunk_planes, c++) {
            const int64_t cz = std::min(chunk_planes, nz - z);
            uint8_t *st = b.stage[c & 1];
            const uint8_t *src = direct_in ? direct_in + z * plane : b.h_in;
            if (!direct_in) {
                if ((e = cudaStreamSynchronize(b.cs)) != cudaSuccess) return set_cuda_error(e, "mask upload");
                int rc = read(z, cz, b.h_in);
                if (rc) return rc;
            }
            if ((e = cudaMemcpyAsync(st, src, cz * plane, cudaMemcpyHostToDevice, ust)) != cudaSuccess ||
                (e = launch_bitpack_encode(st, cz * plane, b.packed + z * plane / 32, false, ust)) != cudaSuccess ||
                (overlap_upload && (e = cudaEventRecord(b.up[c], ust)) != cudaSuccess))
                return set_cuda_error(e, "mask upload");
        }
    }

    int rc = MAXI_OK;
    bool pending_write = false;  // pageable output: planes of the last download still to hand to `write`
    int64_t pw_z0 = 0, pw_n = 0;
    auto flush_write = [&]() -> int {
        if (!pending_write) return MAXI_OK;
        cudaError_t ee = cudaEventSynchronize(b.freed);
        if (ee != cudaSuccess) return set_cuda_error(ee, "slab download");
        pending_write = false;
        return write(pw_z0, pw_n, b.h_out);
    };
    bool first_download = true;
    for (int64_t round = 0; round < rounds; round++) {
        const int64_t r0 = round * k, kr = std::max<int64_t>(0, std::min(k, repititions - r0));
        const bool last_round = round + 1 == rounds;
        const int64_t H = std::min(nz, kr * radius);
        const float *d_in_field = round > 0 ? d_field[(round - 1) & 1] : nullptr;
        float *h_out_field = exchange && !last_round ? b.h_field[round & 1] : nullptr;
        for (int64_t s = 0; s < n_slabs; s++) {
            const int64_t z0 = s * S, z1 = std::min(nz, z0 + S);
            const int64_t e0 = std::max<int64_t>(0, z0 - H), e1 = std::min(nz, z1 + H);
            const int64_t ez = e1 - e0;
            if (verbose >= 1)
                printf("\rRound %lld/%lld, slab %lld/%lld", (long long) (round + 1), (long long) rounds,
                       (long long) (s + 1), (long long) n_slabs), fflush(stdout);
            const void *mask_ptr;
            int32_t mask_fmt;
            if (resident) {
                // the chunks holding planes [e0, e1) are packed (all of them after the first round)
                if (overlap_upload && round == 0 &&
                    (e = cudaStreamWaitEvent(b.cs, b.up[(e1 - 1) / chunk_planes], 0)) != cudaSuccess)
                    return set_cuda_error(e, "mask upload");
                mask_ptr = b.packed + e0 * plane / 32;
                mask_fmt = MAXI_MASK_BITPACKED;
            } else {
                // the per-slab mask buffer is free once the previous slab's work is done
                if ((e = cudaStreamSynchronize(b.cs)) != cudaSuccess) return set_cuda_error(e, "out-of-core slab");
                const uint8_t *src = direct_in ? direct_in + e0 * plane : b.h_in;
                if (!direct_in && (rc = read(e0, ez, b.h_in))) return rc;
                if ((e = cudaMemcpyAsync(b.d_mask, src, ez * plane, cudaMemcpyHostToDevice, b.cs)) != cudaSuccess)
                    return set_cuda_error(e, "slab upload");
                mask_ptr = b.d_mask;
                mask_fmt = MAXI_MASK_U8;
            }
            // Repetition j of the round runs on the planes at least (j + 1) x radius
            // from a cut side; the last one's window is [lo_last, hi_last).
            RunOpts o;
            o.shrink_lo = e0 > 0 ? radius : 0;
            o.shrink_hi = e1 < nz ? radius : 0;
            const int64_t lo_last = shrinks ? std::min(ez - 1, o.shrink_lo * std::max<int64_t>(0, kr - 1)) : 0;
            const int64_t hi_last = shrinks ? std::max(lo_last + 1, ez - o.shrink_hi * std::max<int64_t>(0, kr - 1)) : ez;
            if (hi_last - lo_last > win)
                return set_error(MAXI_ERR_CUDA, "internal: output window of %lld planes exceeds %lld",
                                 (long long) (hi_last - lo_last), (long long) win);
            o.init_field = d_in_field ? d_in_field + e0 * plane : nullptr;
            o.final_wait = first_download ? nullptr : b.freed;  // the window buffers' previous copy-out
            uint16_t *out = last_round ? b.d_out - lo_last * plane : nullptr;
            float *fout = last_round ? nullptr : b.d_fwin - lo_last * plane;
            rc = diffusion_device_shrinking(mask_ptr, mask_fmt, ez, ny, nx, kernel, kernel_size, kr, out, fout,
                                            field_type, flags, b.ws, ws_bytes, b.cs, o);
            if (rc) return rc;
            if ((e = cudaEventRecord(b.ready, b.cs)) != cudaSuccess) return set_cuda_error(e, "out-of-core slab");
            // The previous slab's pageable output goes to the writer while this
            // slab computes (its staging buffer is refilled only below).
            if ((rc = flush_write())) return rc;
            if ((e = cudaStreamWaitEvent(b.ds, b.ready, 0)) != cudaSuccess) return set_cuda_error(e, "slab download");
            const int64_t core_off = (z0 - e0 - lo_last) * plane;
            if (last_round) {
                uint16_t *dst = direct_out ? direct_out + z0 * plane : b.h_out;
                e = cudaMemcpyAsync(dst, b.d_out + core_off, (z1 - z0) * plane * 2, cudaMemcpyDeviceToHost, b.ds);
                if (!direct_out) {
                    pending_write = true;
                    pw_z0 = z0;
                    pw_n = z1 - z0;
                }
            } else {
                e = cudaMemcpyAsync(h_out_field + z0 * plane, b.d_fwin + core_off, (z1 - z0) * plane * 4,
                                    cudaMemcpyDeviceToHost, b.ds);
            }
            if (e != cudaSuccess || (e = cudaEventRecord(b.freed, b.ds)) != cudaSuccess)
                return set_cuda_error(e, "slab download");
            first_download = false;
        }
        // The next round reads this round's host field: all copies must have landed.
        if ((e = cudaStreamSynchronize(b.ds)) != cudaSuccess || (e = cudaStreamSynchronize(b.cs)) != cudaSuccess)
            return set_cuda_error(e, "out-of-core round");
    }
    if ((rc = flush_write())) return rc;
    if (verbose >= 1) printf("\rOut-of-core diffusion is complete!\n");
    return MAXI_OK;
}

}  // namespace maxi

extern "C" int maxi_diffusion_out_of_core_ex(const uint8_t *voxels, int64_t nz, int64_t ny, int64_t nx,
                                             int64_t slab_z, const float *kernel, int64_t kernel_size,
                                             int64_t repititions, uint16_t *output, int32_t field_type,
                                             int32_t flags, int verbose) {
    clear_error();
    int rc = validate_common(voxels, nz, ny, nx, kernel, kernel_size, repititions);
    if (rc) return rc;
    if (!output) return set_error(MAXI_ERR_INVALID_ARGUMENT, "output is NULL");
    if (slab_z < 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "slab depth %lld is negative", (long long) slab_z);
    if ((rc = require_device())) return rc;
    const int64_t plane = ny * nx;
    PlaneReader read = [&](int64_t z0, int64_t nzp, uint8_t *dst) {
        memcpy(dst, voxels + z0 * plane, (size_t) (nzp * plane));
        return MAXI_OK;
    };
    PlaneWriter write = [&](int64_t z0, int64_t nzp, const uint16_t *src) {
        memcpy(output + z0 * plane, src, (size_t) (nzp * plane * 2));
        return MAXI_OK;
    };
    return run_slabs(nz, ny, nx, slab_z, kernel, kernel_size, repititions, field_type, flags, verbose, read, write,
                     is_pinned(voxels) ? voxels : nullptr, is_pinned(output) ? output : nullptr);
}

// On-disk form: replaces NS::diffusion_on_disk (src/lib/cpp/include/diffusion.hh:55,
// GPU body src/lib/cpp/gpu/diffusion.cc:808-945) behind the pybind overload
// src/pybind/diffusion-pybind.cc:67-77.  Reads a raw uint8 volume file and
// writes a raw uint16 file, streaming z-slabs of global_z planes (plus deep
// halos) so neither the host nor the device needs the whole volume.  As in the
// reference, the mask of each repetition is rebuilt from the field
// (`field == 1.0f`, src/lib/cpp/gpu/diffusion.cc:885 / store_mask) and the
// field is FP32; no temporary files are written.
extern "C" int maxi_diffusion_on_disk(const char *input_file, const float *kernel, int64_t kernel_size,
                                      const char *output_file, int64_t total_z, int64_t total_y, int64_t total_x,
                                      int64_t global_z, int64_t global_y, int64_t global_x, int64_t repititions,
                                      int verbose) {
    clear_error();
    if (!input_file || !output_file) return set_error(MAXI_ERR_INVALID_ARGUMENT, "file name is NULL");
    const uint8_t dummy = 0;
    int rc = validate_common(&dummy, total_z, total_y, total_x, kernel, kernel_size, repititions);
    if (rc) return rc;
    if (global_z <= 0 || global_y <= 0 || global_x <= 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "global_shape must be positive");
    const int64_t plane = total_y * total_x, n = total_z * plane;
    FILE *fin = fopen(input_file, "rb");
    if (!fin) return set_error(MAXI_ERR_IO, "could not open file: %s", input_file);
    if (fseeko(fin, 0, SEEK_END) != 0 || ftello(fin) < n) {
        fclose(fin);
        return set_error(MAXI_ERR_IO, "%s holds fewer than %lld bytes", input_file, (long long) n);
    }
    if ((rc = require_device())) {
        fclose(fin);
        return rc;
    }
    FILE *fout = fopen(output_file, "wb");
    if (!fout) {
        fclose(fin);
        return set_error(MAXI_ERR_IO, "could not open file: %s", output_file);
    }
    PlaneReader read = [&](int64_t z0, int64_t nzp, uint8_t *dst) {
        if (fseeko(fin, (off_t) (z0 * plane), SEEK_SET) != 0 ||
            fread(dst, 1, (size_t) (nzp * plane), fin) != (size_t) (nzp * plane))
            return set_error(MAXI_ERR_IO, "could not read planes %lld..%lld of %s", (long long) z0,
                             (long long) (z0 + nzp), input_file);
        return (int) MAXI_OK;
    };
    PlaneWriter write = [&](int64_t z0, int64_t nzp, const uint16_t *src) {
        if (fseeko(fout, (off_t) (z0 * plane * 2), SEEK_SET) != 0 ||
            fwrite(src, 2, (size_t) (nzp * plane), fout) != (size_t) (nzp * plane))
            return set_error(MAXI_ERR_IO, "could not write planes %lld..%lld of %s", (long long) z0,
                             (long long) (z0 + nzp), output_file);
        return (int) MAXI_OK;
    };
    rc = run_slabs(total_z, total_y, total_x, global_z, kernel, kernel_size, repititions, MAXI_FIELD_F32,
                   MAXI_FLAG_MASK_FROM_FIELD, verbose, read, write, nullptr, nullptr);
    fclose(fin);
    if (fclose(fout) != 0 && rc == MAXI_OK) rc = set_error(MAXI_ERR_IO, "could not close %s", output_file);
    return rc;
}

// Replaces NS::diffusion_out_of_core (src/lib/cpp/include/diffusion.hh:74):
// global_shape gives the slab depth (global_z); the slabs span the full y and
// x extent, so global_y / global_x only have to be positive.
extern "C" int maxi_diffusion_out_of_core(const uint8_t *voxels, int64_t total_z, int64_t total_y, int64_t total_x,
                                          int64_t global_z, int64_t global_y, int64_t global_x, const float *kernel,
                                          int64_t kernel_size, int64_t repititions, uint16_t *output, int verbose) {
    if (global_y <= 0 || global_x <= 0) {
        clear_error();
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "global_shape must be positive");
    }
    return maxi_diffusion_out_of_core_ex(voxels, total_z, total_y, total_x, global_z, kernel, kernel_size,
                                         repititions, output, MAXI_FIELD_F32, 0, verbose);
}

extern "C" int maxi_out_of_core_plan(int64_t nz, int64_t ny, int64_t nx, int64_t slab_z, int64_t kernel_size,
                                     int64_t repititions, int32_t field_type, int32_t flags, int64_t device_bytes,
                                     int64_t *slab_planes, int64_t *reps_per_round, int32_t *resident_mask) {
    clear_error();
    const uint8_t dummy = 0;
    const float kdummy = 0.0f;
    int rc = validate_common(&dummy, nz, ny, nx, &kdummy, kernel_size, repititions);
    if (rc) return rc;
    if (slab_z < 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "slab depth %lld is negative", (long long) slab_z);
    if (maxi_diffusion_workspace_size(1, ny, nx, field_type) < 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "unknown field_type %d", field_type);
    if (!slab_planes || !reps_per_round || !resident_mask)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "NULL result pointer");
    if (device_bytes <= 0) {
        if ((rc = require_device())) return rc;
        size_t free_b = 0, total_b = 0;
        cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
        if (e != cudaSuccess) return set_cuda_error(e, "cudaMemGetInfo");
        device_bytes = device_budget(free_b);
    }
    const SlabPlan pl = full_plan(nz, ny, nx, slab_z, kernel_size, repititions, field_type, flags, device_bytes,
                                  host_budget());
    *slab_planes = pl.S;
    *reps_per_round = std::min(pl.k, std::max<int64_t>(1, repititions));
    *resident_mask = pl.resident ? 1 : 0;
    if (pl.S < 1 && pl.host_limited)
        return set_error(MAXI_ERR_OUT_OF_MEMORY,
                         "no slab with %lld-plane halos fits %lld device bytes, and exchange rounds need %lld bytes "
                         "of pinned host memory where %lld may be pinned",
                         (long long) std::min(nz, std::max<int64_t>(1, repititions) * (kernel_size / 2)),
                         (long long) device_bytes, (long long) (8 * nz * ny * nx), (long long) host_budget());
    if (pl.S < 1) return set_error(MAXI_ERR_OUT_OF_MEMORY, "no slab fits %lld device bytes", (long long) device_bytes);
    return MAXI_OK;
}
