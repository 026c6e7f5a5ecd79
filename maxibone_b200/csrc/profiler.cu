// Per-kind kernel timing (see profiler.h) and its C ABI.
#include <mutex>
#include <vector>

#include "host_util.h"
#include "profiler.h"

namespace maxi {

namespace {
struct Record {
    int kind;
    cudaEvent_t start, stop;
};
std::mutex g_mu;
bool g_on = false;
std::vector<Record> g_records;
std::vector<cudaEvent_t> g_free;
}  // namespace

bool profiling_enabled() {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_on;
}

cudaEvent_t profile_event() {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_free.empty()) {
        cudaEvent_t e = g_free.back();
        g_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void profile_record(int kind, cudaEvent_t start, cudaEvent_t stop) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_records.push_back({kind, start, stop});
}

}  // namespace maxi

using namespace maxi;

extern "C" {

int maxi_profile_enable(int on) {
    clear_error();
    std::lock_guard<std::mutex> lk(g_mu);
    g_on = on != 0;
    return MAXI_OK;
}

int maxi_profile_read(double *ms_by_kind, int64_t *launches_by_kind, int32_t n_kinds) {
    clear_error();
    if (n_kinds < 0 || (n_kinds > 0 && (!ms_by_kind || !launches_by_kind)))
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "bad output arrays");
    std::vector<Record> recs;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        recs.swap(g_records);
    }
    for (int i = 0; i < n_kinds; i++) {
        ms_by_kind[i] = 0.0;
        launches_by_kind[i] = 0;
    }
    int rc = MAXI_OK;
    for (const Record &r : recs) {
        float ms = 0.0f;
        cudaError_t e = cudaEventSynchronize(r.stop);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, r.start, r.stop);
        if (e != cudaSuccess && rc == MAXI_OK) rc = set_cuda_error(e, "profile event");
        if (r.kind >= 0 && r.kind < n_kinds) {
            ms_by_kind[r.kind] += ms;
            launches_by_kind[r.kind] += 1;
        }
    }
    std::lock_guard<std::mutex> lk(g_mu);
    for (const Record &r : recs) {
        g_free.push_back(r.start);
        g_free.push_back(r.stop);
    }
    return rc;
}

}  // extern "C"
