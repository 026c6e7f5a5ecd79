// Batched form: many independent volumes of uneven sizes, each with its own
// kernel and repetition count, run as one CUDA graph.
//
// Plan creation sorts the volumes into groups that share a kernel and a
// repetition count.  A group on the tensor-core path (16-bit field, radius
// <= 32, x extent a multiple of 8 and >= 64) runs each pass of each repetition
// as ONE persistent launch over the tiles of all its volumes (tc_batch.cu);
// the other volumes run their own passes.  The whole repetition loop is
// captured once into a CUDA graph and replayed by maxi_batch_plan_run(): a
// 64-volume, 50-repetition batch is a single graph launch.
//
// Autotuning (MAXI_FLAG_AUTOTUNE): for each tensor-core group the plan times
// three repetitions of each form the group can run in -- one batched
// tensor-core launch per pass over all its volumes, the single-volume
// tensor-core launches volume by volume, and the per-volume CUDA-core passes
// -- and keeps the fastest.  Choices are keyed by the GPU (name and SM count),
// field type, radius and the group's volume shapes, kept for the process and
// persisted in a JSON file (MAXIBONE_TUNE_CACHE, else
// $XDG_CACHE_HOME/maxibone_b200/batch_tune.json or
// ~/.cache/maxibone_b200/batch_tune.json; MAXIBONE_TUNE_CACHE set to an empty
// string keeps them in the process only), so a later process plans without
// timing.  maxi_batch_plan_describe() reports each group's form and timings.
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "host_util.h"
#include "tc_batch.h"
#include "unrolled.h"

extern "C" int64_t maxi_diffusion_workspace_size(int64_t nz, int64_t ny, int64_t nx, int32_t field_type);

namespace maxi {

struct BatchVolume {
    maxi_volume v;
    std::vector<float> kernel;
    int64_t ws_offset = 0;
    int group = -1;  // tensor-core group index, or -1 for the per-volume path
    // Storage type this volume runs in: the plan's, or FP32 for a 16-bit plan's
    // volume whose shape the tensor-core passes do not take (the FP32 form is
    // faster and more accurate than the 16-bit CUDA-core passes), as
    // maxi_diffusion_device() does.
    int32_t run_type = MAXI_FIELD_F32;
};

// How a tensor-core group runs: one launch per pass over all its volumes, the
// single-volume tensor-core launches per volume (separate y and x passes, or
// the fused y + x kernel where the radius allows it), or per-volume CUDA-core
// passes.
enum GroupForm { kFormBatched = 0, kFormPerVolumeTc = 1, kFormPerVolumeFused = 2, kFormCudaCores = 3, kForms = 4 };
static const char *const kFormNames[kForms] = {"batched", "per_volume_tc", "per_volume_fused", "cuda_cores"};

struct TcGroup {
    std::vector<int> members;
    std::vector<float> kernel;
    int64_t reps = 0;
    tc::TcGeometry geo{};
    tc::TcVol *d_vols = nullptr;
    int64_t *d_prefix = nullptr;  // [4][n + 1]: z columns, y columns, x tiles, fused y + x tiles
    int64_t totals[4] = {0, 0, 0, 0};
    int form = kFormBatched;
    std::string note;
};

// A tuning decision and the timings it came from (ms for 3 repetitions; < 0: not timed).
struct TuneEntry {
    int form = kFormBatched;
    float ms[kForms] = {-1.0f, -1.0f, -1.0f, -1.0f};
};

static std::mutex g_tune_mu;
static std::map<std::string, TuneEntry> g_tune_cache;  // group key -> decision
static bool g_tune_loaded = false;

// Path of the persistent tuning cache ("" when persistence is off).
static std::string tune_cache_path() {
    if (const char *env = getenv("MAXIBONE_TUNE_CACHE")) return env;
    const char *xdg = getenv("XDG_CACHE_HOME");
    if (xdg && *xdg) return std::string(xdg) + "/maxibone_b200/batch_tune.json";
    const char *home = getenv("HOME");
    if (home && *home) return std::string(home) + "/.cache/maxibone_b200/batch_tune.json";
    return "";
}

// Reads the cache file into g_tune_cache (entries already in the process win).
// One entry per line: "key": {"form": "name", "batched_ms": t, ...}.
static void tune_load_locked() {
    g_tune_loaded = true;
    const std::string path = tune_cache_path();
    if (path.empty()) return;
    FILE *f = fopen(path.c_str(), "r");
    if (!f) return;
    char line[4096];
    while (fgets(line, sizeof line, f)) {
        const char *k0 = strchr(line, '"');
        const char *k1 = k0 ? strchr(k0 + 1, '"') : nullptr;
        const char *fm = k1 ? strstr(k1, "\"form\": \"") : nullptr;
        if (!fm) continue;
        const std::string key(k0 + 1, k1);
        fm += strlen("\"form\": \"");
        TuneEntry e;
        e.form = -1;
        for (int i = 0; i < kForms; i++) {
            const size_t n = strlen(kFormNames[i]);
            if (strncmp(fm, kFormNames[i], n) == 0 && fm[n] == '"') e.form = i;
            const std::string tag = std::string("\"") + kFormNames[i] + "_ms\": ";
            if (const char *t = strstr(fm, tag.c_str())) e.ms[i] = strtof(t + tag.size(), nullptr);
        }
        if (e.form >= 0 && !g_tune_cache.count(key)) g_tune_cache[key] = e;
    }
    fclose(f);
}

// Writes g_tune_cache to the cache file (a temporary file renamed over it);
// failures leave the process cache as it is.
static void tune_save_locked() {
    const std::string path = tune_cache_path();
    if (path.empty()) return;
    for (size_t i = 1; i < path.size(); i++)  // mkdir -p of the directory
        if (path[i] == '/') mkdir(path.substr(0, i).c_str(), 0755);
    const std::string tmp = path + ".tmp" + std::to_string((long long) getpid());
    FILE *f = fopen(tmp.c_str(), "w");
    if (!f) return;
    fprintf(f, "{\n\"format\": \"maxibone_b200 batch tuning cache 1\",\n\"entries\": {\n");
    size_t i = 0;
    for (const auto &kv : g_tune_cache) {
        fprintf(f, "\"%s\": {\"form\": \"%s\"", kv.first.c_str(), kFormNames[kv.second.form]);
        for (int j = 0; j < kForms; j++)
            if (kv.second.ms[j] >= 0.0f) fprintf(f, ", \"%s_ms\": %.4f", kFormNames[j], kv.second.ms[j]);
        fprintf(f, "}%s\n", ++i < g_tune_cache.size() ? "," : "");
    }
    fprintf(f, "}\n}\n");
    const bool ok = fclose(f) == 0;
    if (!ok || rename(tmp.c_str(), path.c_str()) != 0) remove(tmp.c_str());
}

}  // namespace maxi

struct maxi_batch_plan {
    int device = 0;
    int32_t field_type = 0, flags = 0;
    std::vector<maxi::BatchVolume> vols;
    std::vector<maxi::TcGroup> groups;
    char *d_ws = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::string description;
};

namespace maxi {

static size_t field_size(int32_t ft) { return ft == MAXI_FIELD_F32 ? 4 : 2; }

template <typename S>
static S *vol_buf(maxi_batch_plan *p, const BatchVolume &bv, int b) {
    const int64_t n = bv.v.nz * bv.v.ny * bv.v.nx;
    return reinterpret_cast<S *>(p->d_ws + bv.ws_offset + b * round_up((int64_t) sizeof(S) * n, 256));
}
static uint32_t *vol_packed(maxi_batch_plan *p, const BatchVolume &bv) {
    const int64_t n = bv.v.nz * bv.v.ny * bv.v.nx;
    return reinterpret_cast<uint32_t *>(p->d_ws + bv.ws_offset + 2 * round_up((int64_t) field_size(bv.run_type) * n, 256));
}

// Enqueues mask packing and the rep-0 field of every member volume.
template <typename S>
static cudaError_t enqueue_init(maxi_batch_plan *p, const std::vector<int> &idx, cudaStream_t st) {
    for (int i : idx) {
        BatchVolume &bv = p->vols[i];
        const int64_t n = bv.v.nz * bv.v.ny * bv.v.nx;
        cudaError_t e = launch_bitpack_encode(static_cast<const uint8_t *>(bv.v.mask), n, vol_packed(p, bv), false, st);
        if (e == cudaSuccess) e = launch_init_field<S>(vol_packed(p, bv), MAXI_MASK_BITPACKED, vol_buf<S>(p, bv, 0), n, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// The per-volume path of one volume (all repetitions).  fused: the y and x
// passes as the fused kernel where it applies (else two kernels, the form of
// the batched launches).
template <typename S>
static cudaError_t enqueue_single(maxi_batch_plan *p, BatchVolume &bv, int32_t extra_flags, cudaStream_t st,
                                  bool fused = false) {
    const int64_t n = bv.v.nz * bv.v.ny * bv.v.nx;
    cudaError_t e = launch_bitpack_encode(static_cast<const uint8_t *>(bv.v.mask), n, vol_packed(p, bv), false, st);
    if (e != cudaSuccess) return e;
    const Volume vol{bv.v.nz, bv.v.ny, bv.v.nx};
    // The batched tensor-core launches run the y and x passes as separate
    // kernels; the per-volume path does the same unless asked for the fused
    // kernel (a group's chosen form applies to all its volumes).
    return dispatch_unrolled<S>(vol, vol_packed(p, bv), MAXI_MASK_BITPACKED, bv.kernel.data(),
                                (int) (bv.v.kernel_size / 2), bv.v.repititions, vol_buf<S>(p, bv, 0),
                                vol_buf<S>(p, bv, 1), bv.v.output, bv.v.field_out,
                                p->flags | extra_flags | (fused ? 0 : MAXI_FLAG_SEPARATE_PASSES), st);
}

// All repetitions of a tensor-core group as batched launches.
template <typename S>
static cudaError_t enqueue_group_tc(maxi_batch_plan *p, TcGroup &g, cudaStream_t st) {
    // A group of one volume runs the single-volume tensor-core launches (tensor
    // maps as kernel parameters instead of a device table); the arithmetic per
    // tile is the same.
    if (g.members.size() == 1) return enqueue_single<S>(p, p->vols[g.members[0]], 0, st, false);
    cudaError_t e = enqueue_init<S>(p, g.members, st);
    if (e != cudaSuccess) return e;
    const bool bf16 = std::is_same<S, __nv_bfloat16>::value;
    const bool ef = (p->flags & MAXI_FLAG_NEAREST_ROUNDING) == 0 && g.geo.radius >= 4;
    const bool hi_only = tc::tc_single_set(g.geo.radius, (p->flags & MAXI_FLAG_SPLIT_COEFFICIENTS) != 0);
    const int n = (int) g.members.size();
    // The y and x passes as the fused kernel where it applies (one coefficient
    // set, radius <= 32), as the single-volume call runs them.
    const bool fused = hi_only && (p->flags & MAXI_FLAG_SEPARATE_PASSES) == 0 && g.geo.radius <= tc::kTcMaxRadius;
    int in = 0;
    for (int64_t rep = 0; rep < g.reps; rep++) {
        const bool last = rep + 1 == g.reps;
        if (fused) {
            // z: buffer in -> in ^ 1 ([z][y][x]); fused y + x: in ^ 1 -> in ([y][z][x] rows).
            if ((e = tc::tc_batch_pass(g.d_vols, g.d_prefix, g.totals[0], n, 0, in, false, g.kernel.data(), g.geo, bf16, ef, rep > 0, st, hi_only)) != cudaSuccess ||
                (e = tc::tc_batch_pass(g.d_vols, g.d_prefix + 3 * (n + 1), g.totals[3], n, 3, in ^ 1, last, g.kernel.data(), g.geo, bf16, ef, true, st, hi_only)) != cudaSuccess)
                return e;
            continue;
        }
        // The x pass hands the next repetition its field in [y][z][x] row order.
        if ((e = tc::tc_batch_pass(g.d_vols, g.d_prefix, g.totals[0], n, 0, in, false, g.kernel.data(), g.geo, bf16, ef, rep > 0, st, hi_only)) != cudaSuccess ||
            (e = tc::tc_batch_pass(g.d_vols, g.d_prefix + (n + 1), g.totals[1], n, 1, in ^ 1, false, g.kernel.data(), g.geo, bf16, ef, false, st, hi_only)) != cudaSuccess ||
            (e = tc::tc_batch_pass(g.d_vols, g.d_prefix + 2 * (n + 1), g.totals[2], n, 2, in, last, g.kernel.data(), g.geo, bf16, ef, true, st, hi_only)) != cudaSuccess)
            return e;
        in ^= 1;
    }
    return cudaSuccess;
}

// All repetitions of a group in the given form.
template <typename S>
static cudaError_t enqueue_group(maxi_batch_plan *p, TcGroup &g, int form, cudaStream_t st) {
    if (form == kFormBatched) return enqueue_group_tc<S>(p, g, st);
    cudaError_t e = cudaSuccess;
    const int32_t extra = form == kFormCudaCores ? MAXI_FLAG_NO_TENSOR_CORES : 0;
    for (int i : g.members)
        if ((e = enqueue_single<S>(p, p->vols[i], extra, st, form == kFormPerVolumeFused)) != cudaSuccess) break;
    return e;
}

template <typename S>
static cudaError_t enqueue_all(maxi_batch_plan *p, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    for (TcGroup &g : p->groups)
        if ((e = enqueue_group<S>(p, g, g.form, st)) != cudaSuccess) return e;
    for (BatchVolume &bv : p->vols) {
        if (bv.group >= 0) continue;
        e = (sizeof(S) == 2 && bv.run_type == MAXI_FIELD_F32) ? enqueue_single<float>(p, bv, 0, st)
                                                               : enqueue_single<S>(p, bv, 0, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <typename S>
static cudaError_t time_group(maxi_batch_plan *p, TcGroup &g, int form, cudaStream_t st, float *ms) {
    // Three repetitions so the one-off mask packing and field set-up of both
    // candidates do not dominate the comparison.
    const int64_t saved = g.reps;
    std::vector<int64_t> saved_reps;
    g.reps = 3;
    for (int i : g.members) {
        saved_reps.push_back(p->vols[i].v.repititions);
        p->vols[i].v.repititions = 3;
    }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaError_t e = cudaSuccess;
    for (int it = 0; it < 2 && e == cudaSuccess; it++) {  // first run warms up
        cudaEventRecord(a, st);
        e = enqueue_group<S>(p, g, form, st);
        cudaEventRecord(b, st);
    }
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    g.reps = saved;
    for (size_t k = 0; k < g.members.size(); k++) p->vols[g.members[k]].v.repititions = saved_reps[k];
    return e;
}

// Tuning key of a group: GPU name and SM count, field type, radius and the
// sorted volume shapes (z x y x x).
static std::string group_key(const maxi_batch_plan *p, const TcGroup &g) {
    cudaDeviceProp prop;
    std::string gpu = "unknown";
    if (cudaGetDeviceProperties(&prop, p->device) == cudaSuccess)
        gpu = std::string(prop.name) + " sm" + std::to_string(prop.multiProcessorCount);
    else
        cudaGetLastError();
    for (char &c : gpu)
        if (c == '"' || c == '\\' || c == '|') c = '_';
    static const char *const types[] = {"f32", "bf16", "f16", "f64"};
    const int ft = p->field_type;
    std::string s = gpu + "|" + (ft >= 0 && ft < 4 ? types[ft] : "?") + "|r" + std::to_string(g.kernel.size() / 2) + "|";
    std::vector<std::string> shapes;
    for (int i : g.members) {
        const maxi_volume &v = p->vols[i].v;
        shapes.push_back(std::to_string(v.nz) + "x" + std::to_string(v.ny) + "x" + std::to_string(v.nx));
    }
    std::sort(shapes.begin(), shapes.end());
    for (size_t i = 0; i < shapes.size(); i++) s += (i ? "," : "") + shapes[i];
    return s;
}

template <typename S>
static int build_plan(maxi_batch_plan *p, cudaStream_t user_st) {
    const bool tc_type = sizeof(S) == 2 && (p->flags & MAXI_FLAG_NO_TENSOR_CORES) == 0;
    // Group tensor-core-eligible volumes by (kernel, repetitions).
    for (size_t i = 0; i < p->vols.size(); i++) {
        BatchVolume &bv = p->vols[i];
        const int radius = (int) (bv.v.kernel_size / 2);
        const bool eligible = tc_type && bv.v.repititions > 0 && radius <= tc::kTcMaxRadius &&
                              tc::tc_supported(radius, bv.v.nz, bv.v.ny, bv.v.nx) &&
                              ((reinterpret_cast<uintptr_t>(bv.v.output) | reinterpret_cast<uintptr_t>(bv.v.field_out)) & 15) == 0;
        if (!eligible) continue;
        int gi = -1;
        for (size_t k = 0; k < p->groups.size(); k++)
            if (p->groups[k].reps == bv.v.repititions && p->groups[k].kernel == bv.kernel) gi = (int) k;
        if (gi < 0) {
            TcGroup g;
            g.kernel = bv.kernel;
            g.reps = bv.v.repititions;
            g.geo = tc::tc_geometry(radius);
            p->groups.push_back(g);
            gi = (int) p->groups.size() - 1;
        }
        p->groups[gi].members.push_back((int) i);
        bv.group = gi;
    }
    // Default form: one batched launch per pass; a group of one volume runs the
    // single-volume launches with the fused y + x kernel, as a single-volume
    // call does.
    for (TcGroup &g : p->groups) g.form = g.members.size() == 1 ? kFormPerVolumeFused : kFormBatched;
    // Device tables of each group.
    for (TcGroup &g : p->groups) {
        const int n = (int) g.members.size();
        std::vector<tc::TcVol> vols(n);
        std::vector<int64_t> prefix(4 * (n + 1), 0);
        for (int k = 0; k < n; k++) {
            BatchVolume &bv = p->vols[g.members[k]];
            if (tc::tc_fill_volume(vols[k], vol_buf<S>(p, bv, 0), vol_buf<S>(p, bv, 1), vol_packed(p, bv), bv.v.output,
                                   bv.v.field_out, bv.v.nz, bv.v.ny, bv.v.nx, std::is_same<S, __nv_bfloat16>::value,
                                   g.geo) != 0)
                return set_error(MAXI_ERR_CUDA, "could not encode the tensor maps of a batch volume");
            prefix[k + 1] = prefix[k] + vols[k].cols_z;
            prefix[(n + 1) + k + 1] = prefix[(n + 1) + k] + vols[k].cols_y;
            prefix[2 * (n + 1) + k + 1] = prefix[2 * (n + 1) + k] + vols[k].tiles_x;
            prefix[3 * (n + 1) + k + 1] = prefix[3 * (n + 1) + k] + vols[k].tiles_yx;
        }
        for (int q = 0; q < 4; q++) g.totals[q] = prefix[q * (n + 1) + n];
        if (cudaMalloc(&g.d_vols, sizeof(tc::TcVol) * n) != cudaSuccess ||
            cudaMalloc(&g.d_prefix, sizeof(int64_t) * prefix.size()) != cudaSuccess) {
            cudaGetLastError();
            return set_error(MAXI_ERR_OUT_OF_MEMORY, "could not allocate the batch tables");
        }
        if (cudaMemcpy(g.d_vols, vols.data(), sizeof(tc::TcVol) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(g.d_prefix, prefix.data(), sizeof(int64_t) * prefix.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            return set_cuda_error(cudaGetLastError(), "batch table upload");
    }
    // Autotune: the fastest form of each group (from the cache when known).
    if (p->flags & MAXI_FLAG_AUTOTUNE) {
        for (TcGroup &g : p->groups) {
            const std::string key = group_key(p, g);
            bool known = false;
            TuneEntry te;
            {
                std::lock_guard<std::mutex> lk(g_tune_mu);
                if (!g_tune_loaded) tune_load_locked();
                auto it = g_tune_cache.find(key);
                if (it != g_tune_cache.end()) known = true, te = it->second;
            }
            if (!known) {
                // A single volume's batched launch is its per-volume launch.
                te.form = -1;
                for (int f = 0; f < kForms; f++) {
                    if (f == kFormBatched && g.members.size() == 1) continue;
                    cudaError_t e = time_group<S>(p, g, f, user_st, &te.ms[f]);
                    if (e != cudaSuccess) return set_cuda_error(e, "batch autotuning");
                    if (te.form < 0 || te.ms[f] < te.ms[te.form]) te.form = f;
                }
                std::lock_guard<std::mutex> lk(g_tune_mu);
                g_tune_cache[key] = te;
                tune_save_locked();
            }
            g.form = te.form;
            std::string note = known ? "cached choice" : "tuned";
            char buf[96];
            bool first = true;
            for (int f = 0; f < kForms; f++)
                if (te.ms[f] >= 0.0f) {
                    snprintf(buf, sizeof(buf), "%s %s %.3f ms", first ? ":" : ",", kFormNames[f], te.ms[f]);
                    note += buf;
                    first = false;
                }
            note += std::string(" (3 repetitions) -> ") + kFormNames[te.form];
            g.note = note;
        }
    }
    // Capture the whole repetition loop.
    cudaStream_t cap;
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
        return set_cuda_error(cudaGetLastError(), "capture stream");
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaError_t ee = enqueue_all<S>(p, cap);
        e = cudaStreamEndCapture(cap, &p->graph);
        if (ee != cudaSuccess) e = ee;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
    cudaStreamDestroy(cap);
    if (e != cudaSuccess) return set_cuda_error(e, "batch graph capture");
    // Description.
    char line[512];
    snprintf(line, sizeof(line), "%zu volumes, field type %d, %zu tensor-core groups\n", p->vols.size(),
             p->field_type, p->groups.size());
    p->description = line;
    for (size_t k = 0; k < p->groups.size(); k++) {
        const TcGroup &g = p->groups[k];
        snprintf(line, sizeof(line), "group %zu: %zu volumes, kernel length %zu, %lld repetitions, %s%s%s\n", k,
                 g.members.size(), g.kernel.size(), (long long) g.reps,
                 g.form == kFormCudaCores       ? "per-volume CUDA-core passes"
                 : g.form == kFormPerVolumeFused ? "single-volume tensor-core launches, fused y + x where it applies"
                 : g.form == kFormPerVolumeTc || g.members.size() == 1 ? "single-volume tensor-core launches"
                 : tc::tc_single_set(g.geo.radius, (p->flags & MAXI_FLAG_SPLIT_COEFFICIENTS) != 0) &&
                           !(p->flags & MAXI_FLAG_SEPARATE_PASSES) && g.geo.radius <= tc::kTcMaxRadius
                     ? "one tensor-core launch per pass (z, fused y + x)"
                     : "one tensor-core launch per pass (z, y, x)",
                 g.note.empty() ? "" : "; ", g.note.c_str());
        p->description += line;
    }
    size_t singles = 0, fp32 = 0;
    for (const BatchVolume &bv : p->vols) {
        singles += bv.group < 0;
        fp32 += bv.group < 0 && bv.run_type != p->field_type;
    }
    snprintf(line, sizeof(line), "%zu volumes on the per-volume path (%zu in the FP32 form: shapes the tensor-core "
             "passes do not take)\n", singles, fp32);
    p->description += line;
    return MAXI_OK;
}

static void destroy_plan(maxi_batch_plan *p) {
    if (!p) return;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    for (TcGroup &g : p->groups) {
        cudaFree(g.d_vols);
        cudaFree(g.d_prefix);
    }
    cudaFree(p->d_ws);
    delete p;
}

}  // namespace maxi

using namespace maxi;

extern "C" {

int maxi_batch_plan_create(const maxi_volume *volumes, int64_t n_volumes, int32_t field_type, int32_t flags,
                           void *stream, maxi_batch_plan **plan) {
    clear_error();
    if (!plan) return set_error(MAXI_ERR_INVALID_ARGUMENT, "plan is NULL");
    *plan = nullptr;
    if (!volumes || n_volumes <= 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "no volumes");
    if (field_type != MAXI_FIELD_F32 && field_type != MAXI_FIELD_BF16 && field_type != MAXI_FIELD_F16)
        return set_error(MAXI_ERR_UNSUPPORTED, "batched form serves the F32, BF16 and F16 fields");
    if (flags & (MAXI_FLAG_REFERENCE_ROUNDING | MAXI_FLAG_MASK_FROM_FIELD))
        return set_error(MAXI_ERR_UNSUPPORTED, "reference rounding and rebuilt masks are not served in batches");
    int rc;
    for (int64_t i = 0; i < n_volumes; i++) {
        const maxi_volume &v = volumes[i];
        if ((rc = validate_common(v.mask, v.nz, v.ny, v.nx, v.kernel, v.kernel_size, v.repititions, 128))) {
            std::string m = last_error_ref();
            return set_error(rc, "volume %lld: %s", (long long) i, m.c_str());
        }
        if (!v.output && !v.field_out) return set_error(MAXI_ERR_INVALID_ARGUMENT, "volume %lld has no output", (long long) i);
        if (v.repititions == 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "volume %lld has zero repetitions", (long long) i);
    }
    if ((rc = require_device())) return rc;
    auto *p = new maxi_batch_plan();
    cudaGetDevice(&p->device);
    p->field_type = field_type;
    p->flags = flags;
    int64_t total = 0;
    for (int64_t i = 0; i < n_volumes; i++) {
        BatchVolume bv;
        bv.v = volumes[i];
        bv.kernel.assign(volumes[i].kernel, volumes[i].kernel + volumes[i].kernel_size);
        bv.v.kernel = nullptr;  // the plan keeps its own copy
        bv.ws_offset = total;
        bv.run_type = field_type;
        const int radius = (int) (bv.v.kernel_size / 2);
        if (field_type != MAXI_FIELD_F32 && !(flags & MAXI_FLAG_NO_TENSOR_CORES) && radius_bucket(radius) >= 0 &&
            !tc::tc_supported(radius, bv.v.nz, bv.v.ny, bv.v.nx))
            bv.run_type = MAXI_FIELD_F32;
        total += round_up(maxi_diffusion_workspace_size(bv.v.nz, bv.v.ny, bv.v.nx, bv.run_type), 1024);
        p->vols.push_back(bv);
    }
    if (cudaMalloc(&p->d_ws, total) != cudaSuccess) {
        cudaGetLastError();
        destroy_plan(p);
        return set_error(MAXI_ERR_OUT_OF_MEMORY, "could not allocate %lld bytes of batch workspace", (long long) total);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (field_type) {
    case MAXI_FIELD_F32: rc = build_plan<float>(p, st); break;
    case MAXI_FIELD_BF16: rc = build_plan<__nv_bfloat16>(p, st); break;
    default: rc = build_plan<__half>(p, st); break;
    }
    if (rc) {
        destroy_plan(p);
        return rc;
    }
    *plan = p;
    return MAXI_OK;
}

int maxi_batch_plan_run(maxi_batch_plan *plan, void *stream) {
    clear_error();
    if (!plan || !plan->exec) return set_error(MAXI_ERR_INVALID_ARGUMENT, "plan is NULL");
    cudaError_t e = cudaGraphLaunch(plan->exec, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? MAXI_OK : set_cuda_error(e, "batch graph launch");
}

int maxi_batch_plan_describe(const maxi_batch_plan *plan, char *buffer, int64_t buffer_bytes) {
    clear_error();
    if (!plan || !buffer || buffer_bytes <= 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "NULL argument");
    snprintf(buffer, (size_t) buffer_bytes, "%s", plan->description.c_str());
    return MAXI_OK;
}

int maxi_batch_tune_forget(void) {
    clear_error();
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache.clear();
    g_tune_loaded = false;
    return MAXI_OK;
}

int maxi_batch_plan_destroy(maxi_batch_plan *plan) {
    clear_error();
    if (plan) {
        cudaDeviceSynchronize();
        destroy_plan(plan);
    }
    return MAXI_OK;
}

int maxi_diffusion_batched(const maxi_volume *volumes, int64_t n_volumes, int32_t field_type, int32_t flags,
                           void *stream) {
    maxi_batch_plan *plan = nullptr;
    int rc = maxi_batch_plan_create(volumes, n_volumes, field_type, flags, stream, &plan);
    if (rc) return rc;
    rc = maxi_batch_plan_run(plan, stream);
    if (rc == MAXI_OK) {
        cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
        if (e != cudaSuccess) rc = set_cuda_error(e, "batched diffusion");
    }
    maxi_batch_plan_destroy(plan);
    return rc;
}

}  // extern "C"
