// event_log.cpp -- the reference's on-disk event log, written by a reporter:
// necsim/impls/std/src/event_log/recorder.rs (EventLogRecorder) with the
// segment layout of bincode 1.3.3's default encoding (fixed-width little
// endian integers, bool as one byte):
//
//   header  EventLogHeader (event_log/mod.rs:9-18): min_time f64, max_time f64,
//           length u64, with_speciation bool, with_dispersal bool   (26 bytes)
//   events  `length` PackedEvent (necsim/core/src/event.rs:18-28), each
//           global_lineage_reference u64, prior_time f64, event_time f64,
//           origin (x u32, y u32, index u32), target (x, y, index),
//           coalescence u64                                         (56 bytes)
//
// The event kind lives in the sign bits of the times (event.rs:105-160):
// speciation p(-) e(+) with target = origin and coalescence = the lineage;
// dispersal with LineageInteraction::Maybe -- what the Independent
// coalescence sampler always reports (coalescence_sampler/independent.rs:52)
// -- p(+) e(-) with coalescence = the lineage.  Each segment is sorted by
// PackedEvent::cmp (event.rs:256-280) before it is written, segments are
// numbered 0, 1, ... in a directory that must not exist yet.
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/necsim_b200.h"

namespace {

struct Packed {
    uint64_t gref;
    double prior, event;  // signed: the kind encoding
    uint32_t ox, oy, oi, tx, ty, ti;
    uint64_t coalescence;
};

inline uint64_t abs_bits(double v) {
    uint64_t b;
    std::memcpy(&b, &v, 8);
    return b & 0x7fffffffffffffffULL;
}

inline double with_sign(double v, bool negative) {
    uint64_t b;
    std::memcpy(&b, &v, 8);
    b = negative ? (b | 0x8000000000000000ULL) : (b & 0x7fffffffffffffffULL);
    std::memcpy(&v, &b, 8);
    return v;
}

// PackedEvent::cmp: event time, origin, target, prior time (made positive),
// global reference
bool packed_less(const Packed &a, const Packed &b) {
    const uint64_t ea = abs_bits(a.event), eb = abs_bits(b.event);
    if (ea != eb) return ea < eb;
    if (a.ox != b.ox) return a.ox < b.ox;
    if (a.oy != b.oy) return a.oy < b.oy;
    if (a.oi != b.oi) return a.oi < b.oi;
    if (a.tx != b.tx) return a.tx < b.tx;
    if (a.ty != b.ty) return a.ty < b.ty;
    if (a.ti != b.ti) return a.ti < b.ti;
    const uint64_t pa = abs_bits(a.prior), pb = abs_bits(b.prior);
    if (pa != pb) return pa < pb;
    return a.gref < b.gref;
}

template <typename T>
void put(std::string &out, T v) {
    char b[sizeof(T)];
    std::memcpy(b, &v, sizeof(T));  // the host is little endian, as bincode's default
    out.append(b, sizeof(T));
}

}  // namespace

struct necsim_event_log {
    std::string directory;
    uint64_t capacity = 0;
    uint64_t segment = 0;
    bool with_speciation = false, with_dispersal = false;
    std::vector<Packed> buffer;
    std::string error;

    int write_segment() {
        if (buffer.empty()) return NECSIM_OK;
        std::sort(buffer.begin(), buffer.end(), packed_less);
        std::string out;
        out.reserve(26 + buffer.size() * 56);
        put<double>(out, with_sign(buffer.front().event, false));
        put<double>(out, with_sign(buffer.back().event, false));
        put<uint64_t>(out, buffer.size());
        put<uint8_t>(out, with_speciation ? 1 : 0);
        put<uint8_t>(out, with_dispersal ? 1 : 0);
        for (const Packed &e : buffer) {
            put<uint64_t>(out, e.gref);
            put<double>(out, e.prior);
            put<double>(out, e.event);
            put<uint32_t>(out, e.ox);
            put<uint32_t>(out, e.oy);
            put<uint32_t>(out, e.oi);
            put<uint32_t>(out, e.tx);
            put<uint32_t>(out, e.ty);
            put<uint32_t>(out, e.ti);
            put<uint64_t>(out, e.coalescence);
        }
        const std::string path = directory + "/" + std::to_string(segment++);
        FILE *f = std::fopen(path.c_str(), "wb");
        if (!f) {
            error = "cannot write " + path;
            return NECSIM_E_INVALID_ARGUMENT;
        }
        bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
        ok = (std::fclose(f) == 0) && ok;
        buffer.clear();
        if (!ok) {
            error = "short write to " + path;
            return NECSIM_E_INVALID_ARGUMENT;
        }
        return NECSIM_OK;
    }

    int push(const Packed &p) {
        buffer.push_back(p);
        if (buffer.size() >= capacity) return write_segment();
        return NECSIM_OK;
    }
};

namespace {

int log_speciation(void *user, const necsim_speciation_event *ev, uint64_t n) {
    auto *log = static_cast<necsim_event_log *>(user);
    log->with_speciation = true;
    for (uint64_t k = 0; k < n; ++k) {
        const necsim_speciation_event &e = ev[k];
        Packed p{e.global_lineage_reference, with_sign(e.prior_time, true), with_sign(e.event_time, false),
                 e.x, e.y, e.index, e.x, e.y, e.index, e.global_lineage_reference};
        if (log->push(p) != NECSIM_OK) return 1;
    }
    return 0;
}

int log_dispersal(void *user, const necsim_dispersal_event *ev, uint64_t n) {
    auto *log = static_cast<necsim_event_log *>(user);
    log->with_dispersal = true;
    for (uint64_t k = 0; k < n; ++k) {
        const necsim_dispersal_event &e = ev[k];
        Packed p{e.global_lineage_reference, with_sign(e.prior_time, false), with_sign(e.event_time, true),
                 e.x, e.y, e.index, e.target_x, e.target_y, e.target_index, e.global_lineage_reference};
        if (log->push(p) != NECSIM_OK) return 1;
    }
    return 0;
}

int make_dirs(const std::string &path) {
    // the parents may exist; the log directory itself must be new
    for (size_t pos = 1; (pos = path.find('/', pos)) != std::string::npos; ++pos) {
        const std::string part = path.substr(0, pos);
        if (mkdir(part.c_str(), 0777) != 0 && errno != EEXIST) return -1;
    }
    return mkdir(path.c_str(), 0777);
}

}  // namespace

extern "C" {

int necsim_event_log_create(const char *directory, uint64_t segment_capacity, int32_t record_speciation,
                            int32_t record_dispersal, necsim_event_log **out) {
    if (!directory || !*directory || !out || segment_capacity == 0) return NECSIM_E_INVALID_ARGUMENT;
    *out = nullptr;
    std::string dir(directory);
    while (dir.size() > 1 && dir.back() == '/') dir.pop_back();
    if (make_dirs(dir) != 0) return NECSIM_E_INVALID_ARGUMENT;  // exists (start from a clean log) or unwritable
    auto *log = new (std::nothrow) necsim_event_log();
    if (!log) return NECSIM_E_OUT_OF_MEMORY;
    log->directory = dir;
    log->capacity = segment_capacity;
    log->with_speciation = record_speciation != 0;
    log->with_dispersal = record_dispersal != 0;
    *out = log;
    return NECSIM_OK;
}

necsim_reporter necsim_event_log_reporter(necsim_event_log *log) {
    necsim_reporter r;
    r.user = log;
    r.report_speciation = log ? log_speciation : nullptr;
    r.report_dispersal = log ? log_dispersal : nullptr;
    return r;
}

int necsim_event_log_close(necsim_event_log *log) {
    if (!log) return NECSIM_E_INVALID_ARGUMENT;
    int rc = log->write_segment();
    if (log->segment == 0) rmdir(log->directory.c_str());  // no events: leave no empty log behind
    delete log;
    return rc;
}

}  // extern "C"
