// Library runtime: stream, status strings, device workspace cache, host-operand
// staging, the device error flag and optional per-kernel timing.
#include "mbg_internal.cuh"

#include <atomic>
#include <cctype>
#include <map>
#include <mutex>
#include <sstream>
#include <vector>
#include <cstring>
#include <cstdlib>

namespace mbg {

namespace {
std::mutex g_mu;
cudaStream_t g_stream = nullptr;               // mbg_set_stream: the process-wide stream
thread_local cudaStream_t t_stream = nullptr;  // mbg_set_thread_stream: this thread's override
thread_local bool t_stream_on = false;
std::atomic<bool> g_sync{true};
thread_local std::string g_last_error;
std::atomic<int> g_fail_alloc_countdown{0};
std::atomic<int64_t> g_launches{0};

struct DeviceCache {
    // free workspace blocks per stream (size -> block): a block goes back to the
    // pool of the stream its call ran on and is handed out again only to calls on
    // that stream, so its reuse is ordered after its last use by stream order
    std::map<cudaStream_t, std::multimap<size_t, void*>> free_blocks;
    int* err_host = nullptr;                    // mapped pinned flag
    int* err_dev = nullptr;
    cudaStream_t copy_in = nullptr, copy_out = nullptr;  // pipelined host path
};
std::map<int, DeviceCache> g_cache;

struct ProfRecord {
    std::string name;
    cudaEvent_t start, stop;
};
std::atomic<bool> g_prof{false};
std::vector<ProfRecord> g_prof_records;
std::vector<cudaEvent_t> g_event_pool;

cudaEvent_t take_event() {
    if (!g_event_pool.empty()) {
        cudaEvent_t e = g_event_pool.back();
        g_event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

int current_device() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) return -1;
    return d;
}
}  // namespace

Tuning& tuning() {
    static Tuning t;
    return t;
}

cudaStream_t stream() { return t_stream_on ? t_stream : g_stream; }
bool sync_mode() { return g_sync.load(); }

void set_error(const char* what, cudaError_t e) {
    g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    cudaGetLastError();  // clear a sticky launch error so the next call starts clean
}
void set_error_msg(const std::string& msg) { g_last_error = msg; }

int check_launch(const char* name) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_last_error = std::string("launch of ") + name + ": " + cudaGetErrorString(e);
        return MBG_ERR_CUDA;
    }
    count_launch();
    return MBG_OK;
}

void count_launch(int n) { g_launches += n; }

// ---- workspace ---------------------------------------------------------------
Workspace::~Workspace() {
    if (!ptr) return;
    std::lock_guard<std::mutex> lk(g_mu);
    g_cache[current_device()].free_blocks[owner].emplace(bytes, ptr);
    ptr = nullptr;
}

int Workspace::reserve(size_t nbytes) {
    if (nbytes == 0) nbytes = 256;
    if (ptr && bytes >= nbytes) return MBG_OK;
    if (ptr) {  // give back the smaller block
        std::lock_guard<std::mutex> lk(g_mu);
        g_cache[current_device()].free_blocks[owner].emplace(bytes, ptr);
        ptr = nullptr;
    }
    const size_t gran = size_t(2) << 20;
    size_t want = (nbytes + gran - 1) / gran * gran;
    owner = stream();
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceCache& dc = g_cache[current_device()];
    auto& pool = dc.free_blocks[owner];
    auto it = pool.lower_bound(want);
    if (it != pool.end() && it->first <= 2 * want) {
        ptr = it->second;
        bytes = it->first;
        pool.erase(it);
        return MBG_OK;
    }
    int cd = g_fail_alloc_countdown.load();
    if (cd > 0) {
        g_fail_alloc_countdown = cd - 1;
        if (cd == 1) {
            set_error_msg("device workspace allocation failed (injected by mbg_debug_fail_alloc)");
            return MBG_ERR_ALLOC;
        }
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        // drop every stream's cached blocks (cudaFree waits for the device) and retry once
        for (auto& sp : dc.free_blocks)
            for (auto& kv : sp.second) cudaFree(kv.second);
        dc.free_blocks.clear();
        cudaGetLastError();
        e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            set_error("cudaMalloc(workspace)", e);
            return (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? MBG_ERR_NO_DEVICE
                                                                                  : MBG_ERR_ALLOC;
        }
    }
    ptr = p;
    bytes = want;
    return MBG_OK;
}

// ---- operands ---------------------------------------------------------------
bool is_device_pointer(const void* p) {
    if (!p) return false;
    cudaPointerAttributes attr;
    cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

int Operand::prepare(const void* p, i64 r, i64 c, i64 l, size_t e, bool copy_in, bool out) {
    user = p; rows = r; cols = c; ld = l; elem = e; copy_out = out;
    if (r <= 0 || c <= 0) { dev = const_cast<void*>(p); dev_ld = l; return MBG_OK; }
    if (is_device_pointer(p)) { dev = const_cast<void*>(p); dev_ld = l; return MBG_OK; }
    staged = true;
    dev_ld = r;
    MBG_TRY(ws.reserve(size_t(r) * size_t(c) * e));
    dev = ws.ptr;
    if (copy_in) return copy_h2d_2d(dev, size_t(r) * e, p, size_t(l) * e, size_t(r) * e, size_t(c), stream());
    return MBG_OK;
}

int Operand::finish() {
    if (staged && copy_out)
        return copy_d2h_2d(const_cast<void*>(user), size_t(ld) * elem, dev, size_t(rows) * elem, size_t(rows) * elem,
                           size_t(cols), stream(), nullptr);
    return MBG_OK;
}

// ---- a second compute stream per device, and scoped stream overrides ----------------
int aux_stream(cudaStream_t* out) {
    static std::map<int, cudaStream_t> aux;
    std::lock_guard<std::mutex> lk(g_mu);
    cudaStream_t& s = aux[current_device()];
    if (!s) MBG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    *out = s;
    return MBG_OK;
}

StreamScope::StreamScope(cudaStream_t s) : saved(t_stream), saved_on(t_stream_on) {
    t_stream = s;
    t_stream_on = true;
}
StreamScope::~StreamScope() {
    t_stream = saved;
    t_stream_on = saved_on;
}

// ---- copy streams of the pipelined host path ---------------------------------------
int copy_streams(cudaStream_t* in, cudaStream_t* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceCache& dc = g_cache[current_device()];
    if (!dc.copy_in) MBG_CUDA(cudaStreamCreateWithFlags(&dc.copy_in, cudaStreamNonBlocking));
    if (!dc.copy_out) MBG_CUDA(cudaStreamCreateWithFlags(&dc.copy_out, cudaStreamNonBlocking));
    *in = dc.copy_in;
    *out = dc.copy_out;
    return MBG_OK;
}

// ---- device error flag ---------------------------------------------------------
int* device_error_flag() {
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceCache& dc = g_cache[current_device()];
    if (!dc.err_host) {
        if (cudaHostAlloc(&dc.err_host, sizeof(int) * 4, cudaHostAllocMapped) != cudaSuccess) {
            cudaGetLastError();
            dc.err_host = nullptr;
            return nullptr;
        }
        std::memset(dc.err_host, 0, sizeof(int) * 4);
        if (cudaHostGetDevicePointer(&dc.err_dev, dc.err_host, 0) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
    }
    return dc.err_dev;
}

int read_and_clear_device_error() {
    int v = 0, site = 0;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        DeviceCache& dc = g_cache[current_device()];
        if (dc.err_host) {
            volatile int* f = dc.err_host;
            v = f[0];
            site = f[1];
            if (v) {
                f[0] = 0;
                f[1] = 0;
            }
        }
    }
    // the no-allocation entry point's kernels record into a flag of their own
    int site2 = 0;
    const int v2 = noalloc_take_error(&site2);
    if (!v && v2) {
        v = v2;
        site = site2;
    }
    if (v) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "a kernel's bounded wait expired (code %d, site %d); results are invalid", v,
                      site);
        g_last_error = buf;
    }
    return v;
}

int finish_call(bool any_staged) {
    if (any_staged || sync_mode()) {
        MBG_CUDA(cudaStreamSynchronize(stream()));
        if (read_and_clear_device_error()) return MBG_ERR_TIMEOUT;
    }
    return MBG_OK;
}

// ---- timing ------------------------------------------------------------------
ProfScope::ProfScope(const char* name) {
    if (!g_prof.load()) return;
    std::lock_guard<std::mutex> lk(g_mu);
    ProfRecord r{name, take_event(), take_event()};
    cudaEventRecord(r.start, stream());
    g_prof_records.push_back(r);
    slot = int(g_prof_records.size()) - 1;
}
ProfScope::~ProfScope() {
    if (slot < 0) return;
    std::lock_guard<std::mutex> lk(g_mu);
    cudaEventRecord(g_prof_records[slot].stop, stream());
}

}  // namespace mbg

using namespace mbg;

extern "C" {

int mbg_set_stream(void* s) {
    if (g_stream != static_cast<cudaStream_t>(s)) {
        // earlier calls' work finishes first, as when the library had one stream
        if (cudaStreamSynchronize(g_stream) != cudaSuccess) cudaGetLastError();
        g_stream = static_cast<cudaStream_t>(s);
    }
    return MBG_OK;
}
int mbg_set_thread_stream(int on, void* s) {
    t_stream_on = (on != 0);
    t_stream = on ? static_cast<cudaStream_t>(s) : nullptr;
    return MBG_OK;
}
void* mbg_get_stream(void) { return stream(); }
int mbg_set_sync(int on) { g_sync = (on != 0); return MBG_OK; }

int mbg_synchronize(void) {
    MBG_CUDA(cudaStreamSynchronize(stream()));
    if (read_and_clear_device_error()) return MBG_ERR_TIMEOUT;
    return MBG_OK;
}

const char* mbg_status_string(int s) {
    if (s == MBG_OK) return "success";
    if (s > 0) return "invalid argument (Netlib info = position of the argument)";
    switch (s) {
        case MBG_ERR_CUDA: return "CUDA runtime error";
        case MBG_ERR_ALLOC: return "device workspace allocation failed";
        case MBG_ERR_UNSUPPORTED: return "unsupported combination";
        case MBG_ERR_NO_DEVICE: return "no usable CUDA device";
        case MBG_ERR_TIMEOUT: return "kernel wait limit expired";
        case MBG_ERR_INVALID_MODE: return "invalid precision mode or slice count";
        case MBG_ERR_SCRATCH_LIMIT: return "problem exceeds the no-allocation scratch limit";
        default: return "unknown status";
    }
}
const char* mbg_last_error(void) { return g_last_error.c_str(); }
int mbg_version(void) { return 100; }

int mbg_release_workspace(void) {
    MBG_CUDA(cudaStreamSynchronize(stream()));
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto& kv : g_cache) {
        for (auto& sp : kv.second.free_blocks)
            for (auto& b : sp.second) cudaFree(b.second);  // cudaFree waits for the device
        kv.second.free_blocks.clear();
    }
    return MBG_OK;
}

int mbg_prof_enable(int on) { g_prof = (on != 0); return MBG_OK; }

int mbg_prof_reset(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto& r : g_prof_records) {
        g_event_pool.push_back(r.start);
        g_event_pool.push_back(r.stop);
    }
    g_prof_records.clear();
    g_launches = 0;
    return MBG_OK;
}

int mbg_prof_query(const char* sub, double* total_ms, int64_t* launches) {
    std::lock_guard<std::mutex> lk(g_mu);
    double tot = 0.0;
    int64_t cnt = 0;
    for (auto& r : g_prof_records) {
        if (sub && sub[0] && r.name.find(sub) == std::string::npos) continue;
        if (cudaEventSynchronize(r.stop) != cudaSuccess) { cudaGetLastError(); continue; }
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, r.start, r.stop) == cudaSuccess) {
            tot += ms;
            ++cnt;
        } else {
            cudaGetLastError();
        }
    }
    if (total_ms) *total_ms = tot;
    if (launches) *launches = cnt;
    return MBG_OK;
}

int64_t mbg_launch_count(void) { return g_launches.load(); }

// "grouped_simt_tile_<TT>_c<d>" / "grouped_tc_bn_<TT>_c<d>": the per-class entry of a grouped
// sgemm plan's tile table (TT = NN, NT, TN or TT, d = size class 0..4), or nullptr.
static i64* grouped_class_entry(const std::string& k) {
    i64 (*table)[5] = nullptr;
    std::string rest;
    if (k.rfind("grouped_simt_tile_", 0) == 0) { table = tuning().grouped_simt_tile; rest = k.substr(18); }
    else if (k.rfind("grouped_tc_bn_", 0) == 0) { table = tuning().grouped_tc_bn; rest = k.substr(14); }
    else return nullptr;
    if (rest.size() != 5 || rest[2] != '_' || rest[3] != 'c' || rest[4] < '0' || rest[4] > '4') return nullptr;
    const char a = rest[0], b = rest[1];
    if ((a != 'N' && a != 'T') || (b != 'N' && b != 'T')) return nullptr;
    return &table[(a == 'T' ? 2 : 0) + (b == 'T' ? 1 : 0)][rest[4] - '0'];
}

int mbg_set_tuning(const char* key, int64_t value) {
    if (!key) return MBG_ERR_INVALID_MODE;
    const std::string k(key);
    if (i64* e = grouped_class_entry(k)) {
        if (value == 0 || value == 64 || value == 128) { *e = value; return MBG_OK; }
        set_error_msg("tuning value out of range: " + k + " = " + std::to_string(value));
        return MBG_ERR_INVALID_MODE;
    }
    if (k == "trsm_tc_min_k" && value >= 0) { tuning().trsm_tc_min_k = value; return MBG_OK; }
    if (k == "grouped_gemm_tile" && (value == 64 || value == 128)) { tuning().grouped_gemm_tile = value; return MBG_OK; }
    if (k == "trsm_leaf_ctas" && value >= 0) { tuning().trsm_leaf_ctas = value; return MBG_OK; }
    if (k == "trsm_block_rows" && value >= 0 && value <= 1024) { tuning().trsm_block_rows = value; return MBG_OK; }
    if (k == "trsm_block_min_cols" && value >= 0) { tuning().trsm_block_min_cols = value; return MBG_OK; }
    if (k == "trsm_inverse_min_cols" && value >= 0) { tuning().trsm_inverse_min_cols = value; return MBG_OK; }
    if (k == "trsm_inverse_block" && (value == 256 || value == 512)) {
        tuning().trsm_inverse_block = value;
        return MBG_OK;
    }
    if (k == "plain_fp64_simt" && (value == 0 || value == 1)) { tuning().plain_fp64_simt = value; return MBG_OK; }
    if (k == "plain_fp32_staged" && (value == 0 || value == 1)) { tuning().plain_fp32_staged = value; return MBG_OK; }
    if (k == "ozaki_cta_pair" && value >= 0 && value <= 2) { tuning().ozaki_cta_pair = value; return MBG_OK; }
    if (k == "trsm_preslice" && (value == 0 || value == 1)) { tuning().trsm_preslice = value; return MBG_OK; }
    if (k == "ozaki_fused_slicing" && (value == 0 || value == 1)) {
        tuning().ozaki_fused_slicing = value;
        return MBG_OK;
    }
    set_error_msg("unknown tuning key or value: " + k + " = " + std::to_string(value));
    return MBG_ERR_INVALID_MODE;
}

int64_t mbg_get_tuning(const char* key) {
    const std::string k(key ? key : "");
    if (const i64* e = grouped_class_entry(k)) return *e;
    if (k == "trsm_tc_min_k") return tuning().trsm_tc_min_k;
    if (k == "grouped_gemm_tile") return tuning().grouped_gemm_tile;
    if (k == "trsm_leaf_ctas") return tuning().trsm_leaf_ctas;
    if (k == "trsm_block_rows") return tuning().trsm_block_rows;
    if (k == "trsm_block_min_cols") return tuning().trsm_block_min_cols;
    if (k == "trsm_inverse_min_cols") return tuning().trsm_inverse_min_cols;
    if (k == "trsm_inverse_block") return tuning().trsm_inverse_block;
    if (k == "plain_fp64_simt") return tuning().plain_fp64_simt;
    if (k == "plain_fp32_staged") return tuning().plain_fp32_staged;
    if (k == "ozaki_cta_pair") return tuning().ozaki_cta_pair;
    if (k == "ozaki_fused_slicing") return tuning().ozaki_fused_slicing;
    if (k == "trsm_preslice") return tuning().trsm_preslice;
    return -1;
}

// Reads the tuning file: either plain "key value" lines ('#' starts a comment), or
// a JSON object whose top-level members with integer values are applied; string,
// boolean, non-integral and nested (object / array) values are skipped, so a
// file may carry its measurements and a device name beside the keys.  Unknown
// keys and out-of-range values are ignored.  MBG_OK when at least one key was
// applied.
int mbg_load_tuning(const char* path) {
    FILE* f = path ? std::fopen(path, "r") : nullptr;
    if (!f) {
        set_error_msg(std::string("cannot open tuning file ") + (path ? path : "(null)"));
        return MBG_ERR_INVALID_MODE;
    }
    std::string text;
    char buf[4096];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
    std::fclose(f);
    int applied = 0;
    auto apply = [&](const std::string& key, const char* num) {
        char* end = nullptr;
        const long long v = std::strtoll(num, &end, 10);
        const bool integral = end != num && !(*end == '.' || *end == 'e' || *end == 'E');
        if (integral && mbg_set_tuning(key.c_str(), v) == MBG_OK) ++applied;
        return end;
    };
    const size_t first = text.find_first_not_of(" \t\r\n");
    if (first != std::string::npos && text[first] == '{') {
        int depth = 0;
        std::string key;
        bool want_value = false;  // after "key": at depth 1
        for (size_t i = first; i < text.size(); ++i) {
            const char c = text[i];
            if (c == '"') {  // a string: a key, or a value to skip
                std::string str;
                size_t j = i + 1;
                for (; j < text.size() && text[j] != '"'; ++j) {
                    if (text[j] == '\\' && j + 1 < text.size()) ++j;
                    str += text[j];
                }
                i = j;
                if (depth == 1) {
                    if (want_value) key.clear();
                    else key = str;
                    want_value = false;
                }
            } else if (c == '{' || c == '[') {
                if (depth == 1 && want_value) {  // a nested value: skipped with its contents
                    key.clear();
                    want_value = false;
                }
                ++depth;
            } else if (c == '}' || c == ']') {
                --depth;
            } else if (depth != 1) {
                continue;
            } else if (c == ':') {
                want_value = !key.empty();
            } else if (c == ',') {
                key.clear();
                want_value = false;
            } else if (want_value && (c == '-' || std::isdigit((unsigned char)c))) {
                const char* end = apply(key, text.c_str() + i);
                while (*end && (std::isalnum((unsigned char)*end) || *end == '.' || *end == '+' || *end == '-'))
                    ++end;  // the rest of a non-integral number
                i = size_t(end - text.c_str()) - 1;
                key.clear();
                want_value = false;
            } else if (want_value && std::isalpha((unsigned char)c)) {  // true / false / null
                while (i + 1 < text.size() && std::isalpha((unsigned char)text[i + 1])) ++i;
                key.clear();
                want_value = false;
            }
        }
    } else {
        std::istringstream in(text);
        std::string line;
        while (std::getline(in, line)) {
            const size_t hash = line.find('#');
            if (hash != std::string::npos) line.resize(hash);
            std::istringstream ls(line);
            std::string k, v;
            if (!(ls >> k >> v)) continue;
            char* end = nullptr;
            const long long val = std::strtoll(v.c_str(), &end, 10);
            if (end != v.c_str() && *end == '\0' && mbg_set_tuning(k.c_str(), val) == MBG_OK) ++applied;
        }
    }
    return applied > 0 ? MBG_OK : MBG_ERR_INVALID_MODE;
}

int mbg_debug_fail_alloc(int nth) { g_fail_alloc_countdown = nth > 0 ? nth : 0; return MBG_OK; }

}  // extern "C"
