// Host-side infrastructure of the B200 library: error recording, the option
// registry, device buffers and the per-handle CUDA context.
#pragma once
#include "device_alloc.hpp"
#include <cstdlib>
#include <mutex>
#include "../../include/aoclda_b200.h"
#include <cuda_runtime.h>
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace b200 {

// ------------------------------------------------------------------ errors --
// Mirrors the record/warn behaviour of the reference error object
// (source/core/utilities/da_error.hpp:163-260): the last status, message and
// severity of a call are kept in the handle and cleared at the start of the
// next public call.
struct ErrorRecord {
    da_status status = da_status_success;
    da_severity severity = DA_NOTSET;
    std::string message;
    void clear() {
        status = da_status_success;
        severity = DA_NOTSET;
        message.clear();
    }
    da_status error(da_status s, const std::string &m) {
        status = s;
        severity = DA_ERROR;
        message = m;
        return s;
    }
    da_status warn(da_status s, const std::string &m) {
        status = s;
        severity = DA_WARNING;
        message = m;
        return s;
    }
};

// ----------------------------------------------------------------- options --
// A typed registry with the same option names, bounds, defaults and status
// codes as the reference (source/core/utilities/options.hpp:192-940).
enum class LB { m_inf, greaterthan, greaterequal };
enum class UB { p_inf, lessthan, lessequal };
enum class OptKind { Int, Real, String };

struct Option {
    OptKind kind;
    std::string name;
    da_int ival = 0, ilo = 0, ihi = 0;
    double rval = 0, rlo = 0, rhi = 0;
    LB lb = LB::m_inf;
    UB ub = UB::p_inf;
    std::string sval;
    std::vector<std::pair<std::string, da_int>> labels;
};

// trim, squeeze whitespace, lower case (options.hpp:192-202)
inline std::string prep_str(const std::string &in) {
    std::string out;
    bool sp = false;
    for (char c : in) {
        if (std::isspace((unsigned char)c)) {
            sp = true;
            continue;
        }
        if (sp && !out.empty()) out.push_back(' ');
        sp = false;
        out.push_back((char)std::tolower((unsigned char)c));
    }
    return out;
}

// Little byte streams of the model files (da_handle_save_model /
// da_handle_load_model): plain values in host byte order, strings and arrays
// with a 64-bit length; the reader fails (ok = false) instead of reading past
// the end.
struct ByteWriter {
    std::vector<char> b;
    template <typename V> void put(const V &v) {
        const char *p = reinterpret_cast<const char *>(&v);
        b.insert(b.end(), p, p + sizeof(V));
    }
    void put_str(const std::string &s) {
        put<uint64_t>(s.size());
        b.insert(b.end(), s.begin(), s.end());
    }
    template <typename V> void put_vec(const V *p, size_t n) {
        put<uint64_t>(n);
        const char *c = reinterpret_cast<const char *>(p);
        b.insert(b.end(), c, c + n * sizeof(V));
    }
};
struct ByteReader {
    const char *p = nullptr;
    size_t n = 0, pos = 0;
    bool ok = true;
    template <typename V> V get() {
        V v{};
        if (!ok || n - pos < sizeof(V)) {
            ok = false;
            return v;
        }
        std::memcpy(&v, p + pos, sizeof(V));
        pos += sizeof(V);
        return v;
    }
    std::string get_str() {
        const uint64_t len = get<uint64_t>();
        if (!ok || n - pos < len) {
            ok = false;
            return std::string();
        }
        std::string s(p + pos, p + pos + len);
        pos += len;
        return s;
    }
    template <typename V> std::vector<V> get_vec() {
        const uint64_t len = get<uint64_t>();
        std::vector<V> v;
        if (!ok || len > (n - pos) / sizeof(V)) {
            ok = false;
            return v;
        }
        v.resize(len);
        std::memcpy(v.data(), p + pos, len * sizeof(V));
        pos += len * sizeof(V);
        return v;
    }
};

class Registry {
  public:
    std::string errmsg;
    bool single = false; // real options follow float semantics

    void add_int(const std::string &n, da_int lo, LB lb, da_int hi, UB ub, da_int def) {
        Option o;
        o.kind = OptKind::Int;
        o.name = n;
        o.ilo = lo;
        o.ihi = hi;
        o.lb = lb;
        o.ub = ub;
        o.ival = def;
        opts_[n] = o;
    }
    void add_real(const std::string &n, double lo, LB lb, double hi, UB ub, double def) {
        Option o;
        o.kind = OptKind::Real;
        o.name = n;
        o.rlo = lo;
        o.rhi = hi;
        o.lb = lb;
        o.ub = ub;
        o.rval = round_t(def);
        opts_[n] = o;
    }
    void add_string(const std::string &n, std::vector<std::pair<std::string, da_int>> labels,
                    const std::string &def) {
        Option o;
        o.kind = OptKind::String;
        o.name = n;
        o.labels = std::move(labels);
        o.sval = def;
        opts_[n] = o;
    }
    // Re-register an integer option's bounds (kmeans_options.hpp:153-170).
    void rebound_int(const std::string &n, da_int lo, LB lb, da_int hi, UB ub) {
        auto &o = opts_[n];
        o.ilo = lo;
        o.lb = lb;
        o.ihi = hi;
        o.ub = ub;
    }

    da_status set_int(const std::string &name, da_int v) {
        Option *o = find(name);
        if (!o) return da_status_option_not_found;
        if (o->kind != OptKind::Int) return wrong_type(name);
        if (!in_bounds((double)v, (double)o->ilo, o->lb, (double)o->ihi, o->ub)) {
            errmsg = "Option '" + o->name + "': value out-of-bounds";
            return da_status_option_invalid_value;
        }
        o->ival = v;
        return da_status_success;
    }
    da_status set_real(const std::string &name, double v) {
        Option *o = find(name);
        if (!o) return da_status_option_not_found;
        if (o->kind != OptKind::Real) return wrong_type(name);
        v = round_t(v);
        if (!in_bounds(v, o->rlo, o->lb, o->rhi, o->ub)) {
            errmsg = "Option '" + o->name + "': value out-of-bounds";
            return da_status_option_invalid_value;
        }
        o->rval = v;
        return da_status_success;
    }
    da_status set_string(const std::string &name, const std::string &v) {
        Option *o = find(name);
        if (!o) return da_status_option_not_found;
        if (o->kind != OptKind::String) return wrong_type(name);
        for (auto &l : o->labels)
            if (l.first == v) {
                o->sval = v;
                return da_status_success;
            }
        std::string t = prep_str(v);
        for (auto &l : o->labels)
            if (l.first == t) {
                o->sval = t;
                return da_status_success;
            }
        errmsg = "Unrecognized value '" + t + "' for option '" + o->name + "'.";
        return da_status_option_invalid_value;
    }
    da_status get_int(const std::string &name, da_int &v) {
        Option *o = find(name);
        if (!o) return da_status_option_not_found;
        if (o->kind != OptKind::Int) return wrong_type(name);
        v = o->ival;
        return da_status_success;
    }
    da_status get_real(const std::string &name, double &v) {
        Option *o = find(name);
        if (!o) return da_status_option_not_found;
        if (o->kind != OptKind::Real) return wrong_type(name);
        v = o->rval;
        return da_status_success;
    }
    da_status get_string(const std::string &name, std::string &v, da_int *key = nullptr) {
        Option *o = find(name);
        if (!o) return da_status_option_not_found;
        if (o->kind != OptKind::String) return wrong_type(name);
        v = o->sval;
        if (key)
            for (auto &l : o->labels)
                if (l.first == v) *key = l.second;
        return da_status_success;
    }
    // convenience getters for internal use (the option must exist)
    da_int i(const std::string &n) { return opts_.at(n).ival; }
    double r(const std::string &n) { return opts_.at(n).rval; }
    da_int key(const std::string &n) {
        auto &o = opts_.at(n);
        for (auto &l : o.labels)
            if (l.first == o.sval) return l.second;
        return -1;
    }
    // every option's current value (name, kind, value)
    void save(ByteWriter &w) const {
        w.put<uint64_t>(opts_.size());
        for (auto &kv : opts_) {
            const Option &o = kv.second;
            w.put_str(o.name);
            w.put<int32_t>((int32_t)o.kind);
            if (o.kind == OptKind::Int) w.put<int64_t>((int64_t)o.ival);
            else if (o.kind == OptKind::Real) w.put<double>(o.rval);
            else w.put_str(o.sval);
        }
    }
    // values written by save(), through the checking setters; false on a
    // malformed stream, an unknown option or a value the setter rejects
    bool load(ByteReader &r) {
        const uint64_t cnt = r.get<uint64_t>();
        for (uint64_t i = 0; r.ok && i < cnt; ++i) {
            const std::string name = r.get_str();
            const int32_t kind = r.get<int32_t>();
            if (!r.ok) return false;
            Option *o = find(name);
            if (!o || (int32_t)o->kind != kind) return false;
            da_status s;
            if (o->kind == OptKind::Int) s = set_int(name, (da_int)r.get<int64_t>());
            else if (o->kind == OptKind::Real) s = set_real(name, r.get<double>());
            else s = set_string(name, r.get_str());
            if (!r.ok || s != da_status_success) return false;
        }
        return r.ok;
    }
    void print() const {
        for (auto &kv : opts_) {
            const Option &o = kv.second;
            if (o.kind == OptKind::Int)
                std::printf("%s = %lld\n", o.name.c_str(), (long long)o.ival);
            else if (o.kind == OptKind::Real)
                std::printf("%s = %.17g\n", o.name.c_str(), o.rval);
            else
                std::printf("%s = %s\n", o.name.c_str(), o.sval.c_str());
        }
    }

  private:
    std::map<std::string, Option> opts_;
    Option *find(const std::string &name) {
        auto it = opts_.find(name);
        if (it == opts_.end()) it = opts_.find(prep_str(name));
        if (it == opts_.end()) {
            errmsg = "Option '" + prep_str(name) + "' not found in the option registry";
            return nullptr;
        }
        return &it->second;
    }
    da_status wrong_type(const std::string &name) {
        errmsg = "Option setter for '" + name + "' was called with the wrong type";
        return da_status_option_wrong_type;
    }
    double round_t(double v) const { return single ? (double)(float)v : v; }
    // A value is rejected only when a bound comparison holds (options.hpp:
    // 266-276, the setter validating without the NaN check of checkall), so
    // a NaN real value is accepted, as the "outlier target" option needs.
    static bool in_bounds(double v, double lo, LB lb, double hi, UB ub) {
        if (lb == LB::greaterthan && v <= lo) return false;
        if (lb == LB::greaterequal && v < lo) return false;
        if (ub == UB::lessthan && v >= hi) return false;
        if (ub == UB::lessequal && v > hi) return false;
        return true;
    }
};

// Options common to every handle (basic_handle_options.hpp:40-53).
inline void register_common_options(Registry &r) {
    r.add_string("storage order",
                 {{"row-major", row_major},
                  {"column-major", column_major},
                  {"fortran", column_major},
                  {"f", column_major},
                  {"c", row_major}},
                 "column-major");
    r.add_string("check data", {{"yes", 1}, {"no", 0}}, "no");
}

// ---------------------------------------------------------- device buffers --
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    // owner of the allocation; handles that share a buffer (share()) hold it
    // together and the last one frees it
    std::shared_ptr<void> mem;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        mem.reset();
        p = nullptr;
        bytes = 0;
    }
    // grow-only allocation of memory this buffer alone holds (a shared
    // buffer is let go first: whoever calls ensure() writes into it);
    // returns false on failure
    bool ensure(size_t b) {
        if (b <= bytes && p && mem.use_count() == 1) return true;
        release();
        if (b == 0) b = 16;
        void *q = nullptr;
        if (device_alloc(&q, b) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        mem = std::shared_ptr<void>(q, [](void *x) { cudaFree(x); });
        p = q;
        bytes = b;
        return true;
    }
    // hold the same allocation as o (read-only by convention)
    void share(const DevBuf &o) {
        mem = o.mem;
        p = o.p;
        bytes = o.bytes;
    }
    template <typename T> T *as() const { return static_cast<T *>(p); }
};

// Per-handle CUDA context: device, stream, kernel timing.
struct CudaCtx {
    int device = -1;
    cudaStream_t stream = nullptr;     // stream all work is enqueued on
    cudaStream_t own_stream = nullptr; // the handle's own stream
    bool ready = false;
    bool timing = false;
    // Kernel timing: one event pair per timed launch, recorded without
    // synchronising (so that the pair brackets the launch as it runs among
    // its neighbours) and folded into ktime by flush_timing().
    struct TimedLaunch {
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        std::string name;
    };
    std::vector<TimedLaunch> tpool;
    size_t tused = 0;
    std::map<std::string, std::pair<double, long>> ktime; // name -> (ms total, launches)
    std::map<std::string, double> stats;                  // named counters of the last call

    // Lazily bind to the current CUDA device.  Host-only calls (options,
    // argument checks) never need a device; the first call that touches data
    // does.  Fails loudly when no device is present: there is no CPU path.
    da_status init(ErrorRecord &err) {
        if (ready) return da_status_success;
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess || n == 0) {
            cudaGetLastError();
            return err.error(da_status_arch_not_supported,
                             "No CUDA device is available: this library computes on "
                             "NVIDIA B200 (sm_100a) GPUs only.");
        }
        cudaGetDevice(&device);
        if (cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            return err.error(da_status_internal_error, "cudaStreamCreate failed.");
        }
        if (!stream) stream = own_stream;
        ready = true;
        return da_status_success;
    }
    ~CudaCtx() {
        for (auto &t : tpool) {
            if (t.ev0) cudaEventDestroy(t.ev0);
            if (t.ev1) cudaEventDestroy(t.ev1);
        }
        if (own_stream) cudaStreamDestroy(own_stream);
    }
    // Fold the recorded launches into ktime (waits for the last of them).
    void flush_timing() {
        if (tused == 0) return;
        cudaEventSynchronize(tpool[tused - 1].ev1);
        for (size_t i = 0; i < tused; ++i) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, tpool[i].ev0, tpool[i].ev1) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            auto &t = ktime[tpool[i].name];
            t.first += ms;
            t.second += 1;
        }
        tused = 0;
    }
    // Time one launch with events on the handle's stream when timing is on.
    template <typename F> cudaError_t timed(const char *name, F &&launch) {
        if (!timing) return launch();
        if (tused == 1024) flush_timing();
        if (tused == tpool.size()) {
            TimedLaunch t;
            cudaEventCreate(&t.ev0);
            cudaEventCreate(&t.ev1);
            tpool.push_back(t);
        }
        TimedLaunch &t = tpool[tused++];
        t.name = name;
        cudaEventRecord(t.ev0, stream);
        cudaError_t e = launch();
        cudaEventRecord(t.ev1, stream);
        return e;
    }
};

inline da_status cuda_status(ErrorRecord &err, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return da_status_success;
    cudaGetLastError();
    da_status s = (e == cudaErrorMemoryAllocation) ? da_status_memory_error
                                                   : da_status_internal_error;
    return err.error(s, std::string(what) + ": " + cudaGetErrorString(e));
}

#define B200_TRY(expr, what)                                                                   \
    do {                                                                                       \
        cudaError_t _e = (expr);                                                               \
        if (_e != cudaSuccess) return cuda_status(*this->err, _e, what);                       \
    } while (0)

// Validation of a 2-D user array (basic_handle.cpp:110-200 semantics).
template <typename T>
inline da_status check_2d(ErrorRecord &err, da_order order, da_int n_rows, da_int n_cols,
                          const T *data, da_int ld, const char *rn, const char *cn,
                          const char *dn, const char *ldn, da_int rmin = 1, da_int cmin = 1,
                          bool check_nan = false) {
    if (n_rows < rmin)
        return err.error(da_status_invalid_array_dimension,
                         std::string("The function was called with ") + rn + " = " +
                             std::to_string(n_rows) + ". Constraint: " + rn +
                             " >= " + std::to_string(rmin) + ".");
    if (n_cols < cmin)
        return err.error(da_status_invalid_array_dimension,
                         std::string("The function was called with ") + cn + " = " +
                             std::to_string(n_cols) + ". Constraint: " + cn +
                             " >= " + std::to_string(cmin) + ".");
    if (data == nullptr)
        return err.error(da_status_invalid_pointer, std::string("The array ") + dn + " is null.");
    if (order == column_major && ld < n_rows)
        return err.error(da_status_invalid_leading_dimension,
                         std::string("The function was called with ") + rn + " = " +
                             std::to_string(n_rows) + " and " + ldn + " = " +
                             std::to_string(ld) + ". Constraint: " + ldn + " >= " + rn + ".");
    if (order == row_major && ld < n_cols)
        return err.error(da_status_invalid_leading_dimension,
                         std::string("The function was called with ") + cn + " = " +
                             std::to_string(n_cols) + " and " + ldn + " = " +
                             std::to_string(ld) + ". Constraint: " + ldn + " >= " + cn + ".");
    if (check_nan) {
        for (da_int j = 0; j < n_cols; ++j)
            for (da_int i = 0; i < n_rows; ++i) {
                T v = (order == column_major) ? data[i + (size_t)j * ld] : data[(size_t)i * ld + j];
                if (std::isnan(v))
                    return err.error(da_status_invalid_input,
                                     std::string("The array ") + dn +
                                         " contains at least one NaN.");
            }
    }
    return da_status_success;
}

// Copy a user matrix (order, ld) into a device row-major matrix with padded
// width ldo (zero pad columns).  `stage` is scratch for column-major input.
template <typename T>
cudaError_t upload_matrix(da_order order, da_int rows, da_int cols, const T *host, da_int ld,
                          T *dst, int ldo, DevBuf &stage, cudaStream_t s);
template <typename T>
cudaError_t download_matrix(da_order order, da_int rows, da_int cols, const T *dev_rowmajor,
                            int ldi, T *host, da_int ld, DevBuf &stage, cudaStream_t s);

} // namespace b200
