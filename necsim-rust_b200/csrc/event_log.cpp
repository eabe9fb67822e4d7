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
//
// The replay (event_log/replay/*.rs) reads any set of segments back as one
// stream in PackedEvent order: segments are chained into groups of
// time-disjoint segments, the groups merged on their next events.
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
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

// ---- replay: necsim/impls/std/src/event_log/replay/{mod,segment,sorted_segments}.rs ----
namespace {

// A segment read lazily, `capacity` events at a time (segment.rs:35-133).
struct ReplaySegment {
    std::string path;
    FILE *f = nullptr;
    double min_time = 0.0, max_time = 0.0;
    uint64_t length = 0, consumed = 0;
    bool with_speciation = false, with_dispersal = false;
    std::vector<Packed> buf;
    size_t pos = 0;
    uint64_t capacity = 1;

    ~ReplaySegment() {
        if (f) std::fclose(f);
    }

    // the next event, or false at the end (a truncated file ends early, as
    // the reference's failing deserialisation does)
    bool next(Packed &e) {
        if (pos == buf.size()) {
            if (!f || consumed >= length) return false;
            const uint64_t want = std::min<uint64_t>(capacity, length - consumed);
            buf.resize(want);
            const size_t got = std::fread(buf.data(), sizeof(Packed), want, f);
            buf.resize(got);
            consumed += got;
            pos = 0;
            if (got < want) length = consumed;
            if (got == 0) return false;
        }
        e = buf[pos++];
        return true;
    }
};

// A chain of time-disjoint segments read one after the other
// (sorted_segments.rs:41-90), with its next event.
struct ReplayGroup {
    std::vector<ReplaySegment *> segs;
    size_t k = 0;
    Packed next{};
    bool has = false;

    void advance() {
        has = false;
        while (k < segs.size()) {
            if (segs[k]->next(next)) {
                has = true;
                return;
            }
            ++k;
        }
    }
};

struct ReplaySink {
    const necsim_reporter *rep;
    std::vector<necsim_speciation_event> spec;
    std::vector<necsim_dispersal_event> disp;

    int flush() {
        int rc = 0;
        if (!spec.empty() && rep->report_speciation) rc = rep->report_speciation(rep->user, spec.data(), spec.size());
        spec.clear();
        if (rc) return rc;
        if (!disp.empty() && rep->report_dispersal) rc = rep->report_dispersal(rep->user, disp.data(), disp.size());
        disp.clear();
        return rc;
    }

    // PackedEvent -> TypedEvent (event.rs:186-240): prior negative and event
    // positive is a speciation, every other sign pair a dispersal (the
    // interaction the signs encode is not carried by necsim_dispersal_event)
    int push(const Packed &e) {
        const bool prior_neg = std::signbit(e.prior), event_neg = std::signbit(e.event);
        const double prior = with_sign(e.prior, false), event = with_sign(e.event, false);
        if (prior_neg && !event_neg) {
            if (!disp.empty() && flush()) return 1;
            necsim_speciation_event s{};
            s.global_lineage_reference = e.gref;
            s.prior_time = prior;
            s.event_time = event;
            s.x = e.ox;
            s.y = e.oy;
            s.index = e.oi;
            spec.push_back(s);
        } else {
            if (!spec.empty() && flush()) return 1;
            necsim_dispersal_event d{};
            d.global_lineage_reference = e.gref;
            d.prior_time = prior;
            d.event_time = event;
            d.x = e.ox;
            d.y = e.oy;
            d.index = e.oi;
            d.target_x = e.tx;
            d.target_y = e.ty;
            d.target_index = e.ti;
            disp.push_back(d);
        }
        if (spec.size() + disp.size() >= 4096) return flush();
        return 0;
    }
};

int replay_fail(char *err, size_t cap, int code, const std::string &msg) {
    if (err && cap) std::snprintf(err, cap, "%s", msg.c_str());
    return code;
}

}  // namespace

extern "C" int necsim_event_log_replay(const char *const *segments, uint64_t n_segments, uint64_t capacity,
                                       int32_t need_speciation, int32_t need_dispersal, int32_t strict,
                                       const necsim_reporter *reporter, uint64_t *n_events, char *err,
                                       size_t err_cap) {
    if (err && err_cap) err[0] = '\0';
    if (!segments || !reporter || capacity == 0)
        return replay_fail(err, err_cap, NECSIM_E_INVALID_ARGUMENT, "invalid argument");
    if (n_segments == 0)
        return replay_fail(err, err_cap, NECSIM_E_INVALID_ARGUMENT,
                           "The EventLogReplay requires at least one event log segment.");
    try {
        std::vector<std::unique_ptr<ReplaySegment>> owned;
        for (uint64_t j = 0; j < n_segments; ++j) {
            auto s = std::make_unique<ReplaySegment>();
            s->path = segments[j];
            s->capacity = capacity;
            s->f = std::fopen(segments[j], "rb");
            if (!s->f) return replay_fail(err, err_cap, NECSIM_E_INVALID_ARGUMENT, "cannot read " + s->path);
            unsigned char h[26];
            if (std::fread(h, 1, 26, s->f) != 26)
                return replay_fail(err, err_cap, NECSIM_E_INVALID_ARGUMENT, s->path + ": not an event log segment");
            std::memcpy(&s->min_time, h, 8);
            std::memcpy(&s->max_time, h + 8, 8);
            std::memcpy(&s->length, h + 16, 8);
            if (h[24] > 1 || h[25] > 1)
                return replay_fail(err, err_cap, NECSIM_E_INVALID_ARGUMENT, s->path + ": not an event log segment");
            s->with_speciation = h[24] != 0;
            s->with_dispersal = h[25] != 0;
            owned.push_back(std::move(s));
        }
        // every segment reports the same kinds (replay/mod.rs:93-118)
        for (auto &s : owned) {
            if (s->with_speciation != owned[0]->with_speciation)
                return replay_fail(err, err_cap, NECSIM_E_INVALID_ARGUMENT,
                                   "There is a mismatch in reporting speciation events between some segments.");
            if (s->with_dispersal != owned[0]->with_dispersal)
                return replay_fail(err, err_cap, NECSIM_E_INVALID_ARGUMENT,
                                   "There is a mismatch in reporting dispersal events between some segments.");
        }
        // the reporters' needs (rustcoalescence/src/args/cli/replay.rs:61-94)
        const bool ws = owned[0]->with_speciation, wd = owned[0]->with_dispersal;
        std::string need;
        if (need_speciation && !ws && need_dispersal && !wd)
            need = "The reporters require speciation and dispersal events, but the event log cannot provide either.";
        else if (need_speciation && !ws)
            need = "The reporters require speciation events, but the event log cannot provide them.";
        else if (need_dispersal && !wd)
            need = "The reporters require dispersal events, but the event log cannot provide them.";
        if (!need.empty()) {
            if (strict) return replay_fail(err, err_cap, NECSIM_E_INVALID_ARGUMENT, need);
            replay_fail(err, err_cap, NECSIM_OK, need);  // WarnOnly: the message stays as a warning
        }
        // chains of time-disjoint segments (replay/mod.rs:120-164)
        std::vector<ReplaySegment *> rest;
        for (auto &s : owned) rest.push_back(s.get());
        std::vector<std::unique_ptr<ReplayGroup>> groups;
        auto current = std::make_unique<ReplayGroup>();
        double max_time = -INFINITY;
        while (!rest.empty()) {
            double min_time = INFINITY;
            long min_index = -1;
            for (size_t i = 0; i < rest.size(); ++i)
                if (rest[i]->min_time > max_time && rest[i]->min_time < min_time) {
                    min_time = rest[i]->min_time;
                    min_index = (long)i;
                }
            if (min_index < 0) {
                if (current->segs.empty())  // no segment orders after -inf: a NaN or infinite time
                    return replay_fail(err, err_cap, NECSIM_E_INVALID_ARGUMENT,
                                       "event log segment with an invalid minimum time");
                groups.push_back(std::move(current));
                current = std::make_unique<ReplayGroup>();
                max_time = -INFINITY;
                continue;
            }
            ReplaySegment *s = rest[(size_t)min_index];
            rest[(size_t)min_index] = rest.back();  // swap_remove
            rest.pop_back();
            max_time = s->max_time;
            current->segs.push_back(s);
        }
        if (!current->segs.empty()) groups.push_back(std::move(current));
        // k-way merge by PackedEvent::cmp (replay/mod.rs:167-178)
        auto later = [](const ReplayGroup *a, const ReplayGroup *b) { return packed_less(b->next, a->next); };
        std::vector<ReplayGroup *> heap;
        for (auto &g : groups) {
            g->advance();
            if (g->has) heap.push_back(g.get());
        }
        std::make_heap(heap.begin(), heap.end(), later);
        ReplaySink sink{reporter, {}, {}};
        uint64_t count = 0;
        while (!heap.empty()) {
            std::pop_heap(heap.begin(), heap.end(), later);
            ReplayGroup *g = heap.back();
            heap.pop_back();
            if (sink.push(g->next)) return replay_fail(err, err_cap, NECSIM_E_CALLBACK, "a reporter stopped the replay");
            ++count;
            g->advance();
            if (g->has) {
                heap.push_back(g);
                std::push_heap(heap.begin(), heap.end(), later);
            }
        }
        if (sink.flush()) return replay_fail(err, err_cap, NECSIM_E_CALLBACK, "a reporter stopped the replay");
        if (n_events) *n_events = count;
        return NECSIM_OK;
    } catch (const std::bad_alloc &) {
        return replay_fail(err, err_cap, NECSIM_E_OUT_OF_MEMORY, "out of host memory");
    }
}
