// driver.cpp -- `necsim-b200`, a rustcoalescence-style command line front end
// for the B200 backend: reads the reference's RON simulation configuration
// (docs/simulate.ron; rustcoalescence/src/args/config/*), builds the
// scenario, runs it through the C ABI and reports like the reference's
// common plugins (necsim/plugins/common/src/{biodiversity,event_counter,
// execution_time}.rs).
//
//   necsim-b200 simulate <config.ron>   run on the GPU
//   necsim-b200 check <config.ron>      parse and validate, print the run (no GPU)
//   necsim-b200 replay <config.ron>     replay event-log segments through the
//                                       reporters (no GPU)
//
// Supported: speciation; sample (percentage, origin Habitat | List,
// origin Bincode(file), mode Genesis | Resume | Restart(after)); pause (before, config,
// destiny List | Bincode(file), mode Resume | Restart),
// which writes the configuration that resumes the run; rng Seed | Entropy;
// the NonSpatial, SpatiallyImplicit, AlmostInfinite (Circle or Rectangle; Normal or
// Clark2Dt), WrappingNoise and SpatiallyExplicit (habitat, dispersal and turnover maps as (Geo)TIFF files
// or .npy arrays, Uniform(rate) or Map(path) turnover, loading mode FixMe |
// OffByOne | Strict) scenarios; algorithm Independent(...) (Poisson event times)
// or CUDA(...) (exponential event times, the reference CUDA algorithm's
// defaults) with Monolithic, IsolatedIndividuals or IsolatedLandscape parallelism; reporters Biodiversity,
// Counter, Execution, Csv(output), GlobalSpeciation / GlobalTurnover / GlobalCoverage(output)
// (others are ignored with a notice); log EventLog(directory,
// capacity) writes the reference's event log.
#include <fcntl.h>
#include <glob.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <charconv>
#include <chrono>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/necsim_b200.h"
#include "ron.h"

using necsim::ron::Value;

namespace {

struct Fail {
    std::string msg;
};

[[noreturn]] void fail(const std::string &m) { throw Fail{m}; }

// the field `name` of v (a reference into v; field names are literals)
const Value &need(const Value &v, const char *name) {
    const Value *f = v.field(name);
    if (!f) fail("missing field `" + std::string(name) + "` in " + (v.text.empty() ? "(...)" : v.text));
    return *f;
}

// `(a, b)` as two integers
void pair_u64(const Value &v, uint64_t &a, uint64_t &b) {
    if (v.kind != Value::Struct || v.items.size() != 2) fail("expected a pair (a, b)");
    a = v.items[0].as_u64();
    b = v.items[1].as_u64();
}

uint32_t as_u32(const Value &v, const char *what) {
    const uint64_t x = v.as_u64();
    if (x > 0xffffffffULL) fail(std::string(what) + " exceeds 2^32 - 1");
    return (uint32_t)x;
}

// ---- .npy arrays (little-endian, C order) for SpatiallyExplicit maps ----
template <typename T>
std::vector<T> load_npy(const std::string &path, const char *descr, std::vector<uint64_t> &shape) {
    std::ifstream f(path, std::ios::binary);
    if (!f) fail("cannot open " + path);
    char magic[6];
    f.read(magic, 6);
    if (!f || std::memcmp(magic, "\x93NUMPY", 6) != 0) fail(path + ": not a .npy array");
    unsigned char ver[2];
    f.read((char *)ver, 2);
    uint32_t hlen = 0;
    if (ver[0] == 1) {
        unsigned char b[2];
        f.read((char *)b, 2);
        hlen = b[0] | (b[1] << 8);
    } else {
        unsigned char b[4];
        f.read((char *)b, 4);
        hlen = b[0] | (b[1] << 8) | (b[2] << 16) | ((uint32_t)b[3] << 24);
    }
    std::string header(hlen, '\0');
    f.read(&header[0], hlen);
    if (header.find(std::string("'descr': '") + descr + "'") == std::string::npos)
        fail(path + ": expected dtype " + descr);
    if (header.find("'fortran_order': False") == std::string::npos) fail(path + ": expected C order");
    const size_t a = header.find("'shape': (");
    if (a == std::string::npos) fail(path + ": no shape");
    shape.clear();
    std::stringstream ss(header.substr(a + 10, header.find(')', a) - a - 10));
    std::string tok;
    uint64_t total = 1;
    while (std::getline(ss, tok, ',')) {
        if (tok.find_first_not_of(" ") == std::string::npos) continue;
        shape.push_back(std::stoull(tok));
        total *= shape.back();
    }
    std::vector<T> data(total);
    f.read(reinterpret_cast<char *>(data.data()), total * sizeof(T));
    if (!f) fail(path + ": truncated data");
    return data;
}

struct Run {
    necsim_scenario sc{};
    necsim_args args{};
    double speciation = 0.0;
    uint64_t seed = 0;
    bool entropy = false;
    double percentage = 1.0;
    uint32_t rank = 0, size = 1;
    bool landscape = false;  // IsolatedLandscape: partition by subdomain, not by origin index
    std::string csv_output;  // the Csv reporter's file (empty: none)
    // the statistics plugin's GlobalSpeciation, GlobalTurnover and GlobalCoverage files (empty: none)
    std::string speciation_output, turnover_output, coverage_output;
    bool needs_dispersal() const { return rep_counter || !csv_output.empty() || !turnover_output.empty() ||
                                          !coverage_output.empty(); }
    bool needs_speciation() const { return rep_biodiversity || !csv_output.empty() || !speciation_output.empty() ||
                                           !turnover_output.empty(); }
    std::vector<necsim_lineage> list;  // sample origin List
    bool resume = false;
    double pause_before = -1.0;
    double restart_after = 0.0;   // sample mode Restart(after): the resume's minimum event time
    bool restart = false;
    bool pause_restart = false;   // pause mode Restart: the written configuration restarts
    bool listed = false;          // the sample origin lists lineages (List or Bincode)
    std::string pause_bincode;    // pause destiny Bincode(file): the remaining lineages' file
    std::shared_ptr<struct LineageFileSaver> pause_saver;  // that file, created when the config is read
    std::string pause_config;
    std::string algorithm = "Independent";
    bool rep_biodiversity = false, rep_counter = false, rep_execution = false;
    std::string log_directory;  // log: EventLog(directory, capacity)
    uint64_t log_capacity = 1000000;
    std::vector<uint32_t> habitat;
    std::vector<double> dispersal;
    std::vector<double> turnover;  // SpatiallyExplicit turnover map (when given)
    std::string summary;
};

bool ends_with(const std::string &s, const char *suffix) {
    const size_t n = std::strlen(suffix);
    if (s.size() < n) return false;
    for (size_t j = 0; j < n; ++j)
        if (std::tolower((unsigned char)s[s.size() - n + j]) != suffix[j]) return false;
    return true;
}

// a map as a (height, width) array: .npy as stored, anything else as a
// (Geo)TIFF through the library's loader (strict in Strict mode)
template <typename T>
std::vector<T> load_map(const std::string &path, int32_t mode, std::vector<uint64_t> &shape) {
    if (ends_with(path, ".npy")) return load_npy<T>(path, sizeof(T) == 4 ? "<u4" : "<f8", shape);
    void *data = nullptr;
    uint32_t w = 0, h = 0;
    char err[512];
    const int rc = necsim_map_load(path.c_str(), sizeof(T) == 4 ? NECSIM_MAP_U32 : NECSIM_MAP_F64,
                                   mode == NECSIM_MAPS_STRICT ? 1 : 0, &data, &w, &h, err, sizeof(err));
    if (rc) fail(err);
    std::vector<T> out(static_cast<T *>(data), static_cast<T *>(data) + (uint64_t)w * h);
    necsim_map_free(data);
    shape = {h, w};
    return out;
}

// `Rectangle(origin: (x: .., y: ..), width: .., height: ..)` (or its
// `Extent` alias, or the LandscapeExtent wrapped in parentheses): the sample
// extent (necsim/core/src/landscape/extent.rs; width and height 1..=2^32)
void parse_rectangle(const Value &sample, necsim_scenario &sc) {
    const Value *e = &sample;
    if (e->fields.empty() && e->items.size() == 1 && e->items[0].kind == Value::Struct) e = &e->items[0];
    const Value &origin = need(*e, "origin");
    sc.sample_x = as_u32(need(origin, "x"), "origin.x");
    sc.sample_y = as_u32(need(origin, "y"), "origin.y");
    sc.sample_width = need(*e, "width").as_u64();
    sc.sample_height = need(*e, "height").as_u64();
    if (sc.sample_width == 0 || sc.sample_height == 0 || sc.sample_width > (1ULL << 32) ||
        sc.sample_height > (1ULL << 32))
        fail("the sample's width and height must be in 1..=2^32");
}

void parse_scenario(const Value &s, Run &r) {
    const std::string &k = s.variant();
    necsim_scenario &sc = r.sc;
    sc.turnover_rate = 0.5;  // UniformTurnoverRate default
    std::ostringstream o;
    if (k == "NonSpatial") {
        uint64_t w, h;
        pair_u64(need(s, "area"), w, h);
        sc.kind = NECSIM_NON_SPATIAL;
        sc.width = (uint32_t)w;
        sc.height = (uint32_t)h;
        sc.deme = as_u32(need(s, "deme"), "deme");
        o << "NonSpatial(area: (" << w << ", " << h << "), deme: " << sc.deme << ")";
    } else if (k == "SpatiallyImplicit") {
        uint64_t w, h, mw, mh;
        pair_u64(need(s, "local_area"), w, h);
        pair_u64(need(s, "meta_area"), mw, mh);
        sc.kind = NECSIM_SPATIALLY_IMPLICIT;
        sc.width = (uint32_t)w;
        sc.height = (uint32_t)h;
        sc.deme = as_u32(need(s, "local_deme"), "local_deme");
        sc.meta_width = (uint32_t)mw;
        sc.meta_height = (uint32_t)mh;
        sc.meta_deme = as_u32(need(s, "meta_deme"), "meta_deme");
        sc.migration_probability = need(s, "migration").as_f64();
        o << "SpatiallyImplicit(local " << w << "x" << h << "x" << sc.deme << ", meta " << mw << "x" << mh << "x"
          << sc.meta_deme << ", migration " << sc.migration_probability << ")";
    } else if (k == "AlmostInfinite") {
        const Value &sample = need(s, "sample");
        const Value &disp = need(s, "dispersal");
        // almost_infinite/mod.rs:92-122: Circle or Rectangle (alias Extent)
        const bool rectangle = sample.variant() == "Rectangle" || sample.variant() == "Extent";
        if (sample.variant() != "Circle" && !rectangle)
            fail("AlmostInfinite: the sample must be Circle or Rectangle");
        if (disp.variant() != "Normal" && disp.variant() != "Clark2Dt")
            fail("AlmostInfinite: dispersal must be Normal or Clark2Dt");
        sc.kind = disp.variant() == "Normal" ? NECSIM_ALMOST_INFINITE_NORMAL : NECSIM_ALMOST_INFINITE_CLARK2DT;
        if (rectangle) {
            parse_rectangle(sample, sc);
            o << "AlmostInfinite(Rectangle(origin: (" << sc.sample_x << ", " << sc.sample_y
              << "), width: " << sc.sample_width << ", height: " << sc.sample_height << "), ";
        } else {
            // almost_infinite/mod.rs:103-107: the default centre
            sc.centre_x = sc.centre_y = 0x7fffffffu;
            if (const Value *c = sample.field("centre")) {
                sc.centre_x = as_u32(need(*c, "x"), "centre.x");
                sc.centre_y = as_u32(need(*c, "y"), "centre.y");
            }
            const uint64_t radius = need(sample, "radius").as_u64();
            if (radius > 0xffff) fail("AlmostInfinite: the radius is a u16");
            sc.radius = (uint32_t)radius;
            o << "AlmostInfinite(Circle(centre: (" << sc.centre_x << ", " << sc.centre_y << "), radius: " << radius
              << "), ";
        }
        if (sc.kind == NECSIM_ALMOST_INFINITE_NORMAL) {
            sc.sigma = need(disp, "sigma").as_f64();
            o << "Normal(sigma: " << sc.sigma << "))";
        } else {
            sc.shape_u = need(disp, "shape_u").as_f64();
            sc.tail_p = need(disp, "tail_p").as_f64();
            o << "Clark2Dt(shape_u: " << sc.shape_u << ", tail_p: " << sc.tail_p << "))";
        }
    } else if (k == "WrappingNoise") {
        // WrappingNoiseArguments (rustcoalescence/scenarios/src/wrapping_noise.rs:36-56)
        sc.kind = NECSIM_WRAPPING_NOISE;
        sc.noise_seed = need(s, "seed").as_i64();
        sc.coverage = need(s, "coverage").as_f64();
        sc.scale = need(s, "scale").as_f64();
        sc.persistence = need(s, "persistence").as_f64();
        sc.octaves = need(s, "octaves").as_u64();
        const Value &sample = need(s, "sample");
        if (sample.variant() != "Rectangle" && sample.variant() != "Extent")
            fail("WrappingNoise: the sample must be a Rectangle");
        parse_rectangle(sample, sc);
        sc.sigma = need(s, "sigma").as_f64();
        o << "WrappingNoise(seed: " << sc.noise_seed << ", coverage: " << sc.coverage << ", scale: " << sc.scale
          << ", persistence: " << sc.persistence << ", octaves: " << sc.octaves << ", Rectangle(origin: ("
          << sc.sample_x << ", " << sc.sample_y << "), width: " << sc.sample_width << ", height: " << sc.sample_height
          << "), sigma: " << sc.sigma << ")";
    } else if (k == "SpatiallyExplicit") {
        // spatially_explicit/turnover/mod.rs:13-30 (field names and aliases),
        // uniform.rs:131-175 (try_load: the dispersal map first, then the
        // habitat map with the loading mode's fix-ups)
        const Value *hab = s.field("habitat") ? s.field("habitat") : s.field("habitat_map");
        const Value *disp = s.field("dispersal") ? s.field("dispersal") : s.field("dispersal_map");
        if (!hab) fail("missing field `habitat`");
        if (!disp) fail("missing field `dispersal`");
        sc.turnover_rate = 0.5;
        const Value *t = s.field("turnover") ? s.field("turnover") : s.field("turnover_rate");
        const Value *tmap = nullptr;  // Map("path") (turnover/map.rs)
        if (t) {
            const std::string &tv = t->variant();
            if (tv == "Map" && t->items.size() == 1) {
                tmap = &t->items[0];
            } else if ((tv == "Uniform" || tv == "Rate" || tv == "UniformRate") && t->items.size() == 1) {
                sc.turnover_rate = t->items[0].as_f64();
            } else {
                fail("SpatiallyExplicit: turnover must be Uniform(rate) or Map(path)");
            }
        }
        int32_t mode = NECSIM_MAPS_OFF_BY_ONE;  // MapLoadingMode::default (maps/mod.rs:84-88)
        const Value *m = s.field("mode") ? s.field("mode") : s.field("loading_mode");
        if (m) {
            const std::string &mv = m->variant();
            if (mv == "FixMe") mode = NECSIM_MAPS_FIX_ME;
            else if (mv == "OffByOne") mode = NECSIM_MAPS_OFF_BY_ONE;
            else if (mv == "Strict") mode = NECSIM_MAPS_STRICT;
            else fail("SpatiallyExplicit: mode must be FixMe, OffByOne or Strict");
        }
        std::vector<uint64_t> hs, ds, ts;
        r.dispersal = load_map<double>(disp->text, mode, ds);
        if (tmap) r.turnover = load_map<double>(tmap->text, mode, ts);
        r.habitat = load_map<uint32_t>(hab->text, mode, hs);
        if (hs.size() != 2) fail("habitat must be a 2D (height, width) array");
        if (ds.size() != 2) fail("dispersal must be a 2D array");
        if (tmap && ts != hs) fail("the turnover map must have the habitat map's dimensions");
        char err[512];
        const int rc = necsim_maps_fix(r.habitat.data(), (uint32_t)hs[1], (uint32_t)hs[0], r.dispersal.data(), ds[0],
                                       ds[1], tmap ? r.turnover.data() : nullptr, mode, err, sizeof(err));
        if (rc) fail(std::string("SpatiallyExplicit maps: ") + err);
        const uint64_t cells = hs[0] * hs[1];
        if (ds[0] != cells || ds[1] != cells) fail("dispersal must be (cells, cells)");
        sc.kind = NECSIM_SPATIALLY_EXPLICIT;
        sc.height = (uint32_t)hs[0];
        sc.width = (uint32_t)hs[1];
        sc.habitat = r.habitat.data();
        sc.dispersal = r.dispersal.data();
        if (tmap) sc.turnover_map = r.turnover.data();
        o << "SpatiallyExplicit(" << sc.width << "x" << sc.height << " map from " << hab->text
          << (tmap ? ", turnover map " + tmap->text : std::string()) << ")";
    } else {
        fail("scenario " + k + " is not supported by this backend");
    }
    r.summary = o.str();
}

void parse_algorithm(const Value &a, Run &r) {
    const std::string &k = a.variant();
    if (k != "Independent" && k != "CUDA")
        fail("algorithm " + k + " is not the Independent algorithm this backend runs");
    necsim_args &g = r.args;
    if (k == "CUDA") {
        // the CUDA algorithm samples event times with ExpEventTimeSampler
        // (algorithms/cuda/src/launch.rs:121) and defaults delta_t to 3.0 and
        // step_slice to 150 (algorithms/cuda/src/arguments.rs:125-139); its
        // block_size / grid_size defaults are launch shapes of its own kernel
        g.event_time_sampler = NECSIM_SAMPLER_EXP;
        g.delta_t = 3.0;
        g.step_slice = 150;
    }
    r.algorithm = k;
    if (const Value *v = a.field("delta_t")) g.delta_t = v->as_f64();
    if (const Value *v = a.field("step_slice")) g.step_slice = v->as_u64();
    if (const Value *v = a.field("block_size")) g.block_size = as_u32(*v, "block_size");
    if (const Value *v = a.field("grid_size")) g.grid_size = as_u32(*v, "grid_size");
    if (const Value *v = a.field("device")) g.device = (int32_t)as_u32(*v, "device");
    // dedup_cache is accepted: duplicates are removed exactly here, so the
    // reference's lossy cache capacity has no counterpart
    if (const Value *p = a.field("parallelism_mode")) {
        const std::string &m = p->variant();
        if (m == "IsolatedIndividuals" || m == "IsolatedLandscape") {
            const Value &part = need(*p, "partition");
            r.rank = as_u32(need(part, "rank"), "rank");
            r.size = as_u32(need(part, "size"), "size");
            if (r.size == 0 || r.rank >= r.size) fail("the partition rank must be below its size");
            r.landscape = m == "IsolatedLandscape";
        } else if (m != "Monolithic") {
            fail("parallelism mode " + m +
                 " is not supported (Monolithic, IsolatedIndividuals, IsolatedLandscape)");
        }
    }
}

// ---- lineage files (necsim/impls/std/src/lineage_file/{loader,saver}.rs):
// a Vec<Lineage> in bincode 1.3.3's DefaultOptions (`bincode::options()`):
// varint integers (< 251 in one byte, else a 251 / 252 / 253 tag and a u16 /
// u32 / u64, little-endian), f64 as 8 little-endian bytes; a Lineage is
// (global reference u64, last event time f64, x u32, y u32, index u32) ----
void put_varint(std::string &o, uint64_t v) {
    int bytes = 0;
    if (v < 251) {
        o.push_back((char)v);
        return;
    } else if (v <= 0xffffULL) {
        o.push_back((char)251);
        bytes = 2;
    } else if (v <= 0xffffffffULL) {
        o.push_back((char)252);
        bytes = 4;
    } else {
        o.push_back((char)253);
        bytes = 8;
    }
    for (int b = 0; b < bytes; ++b) o.push_back((char)((v >> (8 * b)) & 0xff));
}

uint64_t get_varint(const std::string &in, size_t &at, const std::string &path) {
    if (at >= in.size()) fail(path + ": truncated lineage file");
    const unsigned char tag = (unsigned char)in[at++];
    if (tag < 251) return tag;
    const int bytes = tag == 251 ? 2 : tag == 252 ? 4 : tag == 253 ? 8 : 0;
    if (bytes == 0 || at + bytes > in.size()) fail(path + ": malformed lineage file");
    uint64_t v = 0;
    for (int b = 0; b < bytes; ++b) v |= (uint64_t)(unsigned char)in[at + b] << (8 * b);
    at += bytes;
    return v;
}

std::vector<necsim_lineage> read_lineage_file(const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) fail("cannot read the lineage file " + path);
    const std::string in((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    size_t at = 0;
    const uint64_t n = get_varint(in, at, path);
    if (n > in.size()) fail(path + ": malformed lineage file");
    std::vector<necsim_lineage> out(n);
    for (auto &l : out) {
        l.global_reference = get_varint(in, at, path);
        if (at + 8 > in.size()) fail(path + ": truncated lineage file");
        std::memcpy(&l.last_event_time, in.data() + at, 8);
        at += 8;
        // Lineage::last_event_time is a NonNegativeF64 (lineage.rs:91-106)
        if (!(l.last_event_time >= 0.0)) fail(path + ": a lineage's last event time is negative or NaN");
        const uint64_t x = get_varint(in, at, path), y = get_varint(in, at, path), i = get_varint(in, at, path);
        if ((x | y | i) > 0xffffffffULL) fail(path + ": malformed lineage file");
        l.x = (uint32_t)x;
        l.y = (uint32_t)y;
        l.index = (uint32_t)i;
    }
    // bytes after the list are not read, as bincode::Deserializer::with_reader
    // does not (lineage_file/loader.rs:37-44)
    return out;
}

// LineageFileSaver (necsim/impls/std/src/lineage_file/saver.rs): the file is
// created exclusively when the configuration is read, so an existing file
// fails the run before it simulates, and it is removed again unless the
// lineages are written to it.
struct LineageFileSaver {
    std::string path;
    int fd = -1;
    bool temp = true;

    explicit LineageFileSaver(const std::string &p) : path(p) {
        fd = ::open(p.c_str(), O_WRONLY | O_CREAT | O_EXCL, 0644);
        if (fd < 0) fail("cannot create the lineage file " + p + ": " + std::strerror(errno));
    }
    LineageFileSaver(const LineageFileSaver &) = delete;
    LineageFileSaver &operator=(const LineageFileSaver &) = delete;
    ~LineageFileSaver() {
        if (fd >= 0) ::close(fd);
        if (temp) ::unlink(path.c_str());
    }

    // bincode 1.3.3 DefaultOptions: a varint length, then per lineage the
    // varint global reference, the f64 time as 8 bytes and the varint location
    void write(const std::vector<necsim_lineage> &lins) {
        std::string o;
        put_varint(o, lins.size());
        for (const auto &l : lins) {
            put_varint(o, l.global_reference);
            char t[8];
            std::memcpy(t, &l.last_event_time, 8);
            o.append(t, 8);
            put_varint(o, l.x);
            put_varint(o, l.y);
            put_varint(o, l.index);
        }
        size_t done = 0;
        while (done < o.size()) {
            const ssize_t w = ::write(fd, o.data() + done, o.size() - done);
            if (w <= 0) fail("cannot write the lineage file " + path);
            done += (size_t)w;
        }
        temp = false;
    }
};

void parse_reporters(const Value &root, Run &r);
std::string rust_f64_display(double v);

Run parse_config(const std::string &text) {
    Run r;
    const Value root = necsim::ron::parse(text);
    r.speciation = need(root, "speciation").as_f64();
    if (const Value *s = root.field("sample")) {
        if (const Value *p = s->field("percentage")) r.percentage = p->as_f64();
        if (const Value *o = s->field("origin")) {
            if (o->variant() == "Bincode") {
                r.listed = true;
                r.list = read_lineage_file(need(*o, "file").text);
            } else if (o->variant() == "List") {
                r.listed = true;
                if (o->items.size() != 1 || o->items[0].kind != Value::List) fail("List([...]) expected");
                for (const Value &l : o->items[0].items) {
                    necsim_lineage x{};
                    x.global_reference = need(l, "ref").as_u64();
                    x.last_event_time = need(l, "time").as_f64();
                    if (!(x.last_event_time >= 0.0))
                        fail("a listed lineage's time is negative or NaN (NonNegativeF64)");
                    const Value &loc = need(l, "loc");
                    x.x = as_u32(need(loc, "x"), "x");
                    x.y = as_u32(need(loc, "y"), "y");
                    x.index = as_u32(need(loc, "i"), "i");
                    r.list.push_back(x);
                }
            } else if (o->variant() != "Habitat") {
                fail("sample origin " + o->variant() + " is not supported (Habitat, List, Bincode)");
            }
        }
        if (const Value *m = s->field("mode")) {
            // rustcoalescence/src/cli/simulate/dispatch/valid/launch.rs:60-92: Resume
            // continues with no minimum event time, Restart(after) from `after` on
            if (m->variant() == "Resume") {
                r.resume = true;
            } else if (m->variant() == "Restart") {
                r.resume = r.restart = true;
                r.restart_after = need(*m, "after").as_f64();
                if (!(r.restart_after >= 0.0) || !std::isfinite(r.restart_after))
                    fail("Restart(after) must be a finite time >= 0");
            } else if (m->variant() != "Genesis") {
                fail("sample mode " + m->variant() + " is not supported (Genesis, Resume, Restart)");
            }
        }
    }
    if (r.resume != r.listed) fail("Resume needs a List origin and a List origin needs Resume");
    if (r.restart) {
        // args/config/sample/mod.rs:118-137: every listed lineage lies before
        // the resume point PositiveF64::max_after(after, after)
        const double bound = std::isinf(r.restart_after) ? r.restart_after
                                                          : std::nextafter(r.restart_after, HUGE_VAL);
        for (const necsim_lineage &l : r.list)
            if (l.last_event_time >= bound)
                fail("Lineage #" + std::to_string(l.global_reference) + " at time " +
                     rust_f64_display(l.last_event_time) + " is not before the resume point");
    }
    if (const Value *p = root.field("pause")) {
        if (p->variant() == "Pause") {
            r.pause_before = need(*p, "before").as_f64();
            r.pause_config = need(*p, "config").text;
            if (const Value *d = p->field("destiny")) {
                if (d->variant() == "Bincode") {
                    r.pause_bincode = need(*d, "file").text;
                    r.pause_saver = std::make_shared<LineageFileSaver>(r.pause_bincode);
                }
                else if (d->variant() != "List")
                    fail("pause destiny " + d->variant() + " is not supported (List, Bincode)");
            }
            if (const Value *m = p->field("mode")) {
                if (m->variant() == "Restart")
                    r.pause_restart = true;
                else if (m->variant() != "Resume")
                    fail("pause mode " + m->variant() + " is not supported (Resume, Restart)");
            }
        } else if (p->variant() != "None") {
            fail("pause must be None or Pause(...)");
        }
    }
    if (const Value *lg = root.field("log")) {
        if (lg->variant() == "EventLog") {
            r.log_directory = need(*lg, "directory").text;
            if (const Value *c = lg->field("capacity")) r.log_capacity = c->as_u64();
            if (r.log_capacity == 0) fail("log capacity must be positive");
        } else if (lg->variant() != "None") {
            fail("log must be None or EventLog(...)");
        }
    }
    if (const Value *g = root.field("rng")) {
        if (g->variant() == "Seed" && g->items.size() == 1)
            r.seed = g->items[0].as_u64();
        else if (g->variant() == "Entropy")
            r.entropy = true;
        else
            fail("rng " + g->variant() + " is not supported (Seed(u64), Entropy)");
    } else {
        r.entropy = true;
    }
    parse_scenario(need(root, "scenario"), r);
    r.sc.speciation_probability = r.speciation;
    if (const Value *a = root.field("algorithm")) parse_algorithm(*a, r);
    parse_reporters(root, r);
    r.args.report_dispersal = r.needs_dispersal() ? 1 : 0;
    return r;
}

// reporters: [Plugin(library: .., reporters: [Biodiversity(), ..]), ..]
void parse_reporters(const Value &root, Run &r) {
    if (const Value *reps = root.field("reporters")) {
        std::vector<const Value *> names;
        for (const Value &p : reps->items) {
            if (p.variant() == "Plugin") {
                if (const Value *inner = p.field("reporters"))
                    for (const Value &x : inner->items) names.push_back(&x);
            } else {
                names.push_back(&p);
            }
        }
        for (const Value *n : names) {
            const std::string &v = n->variant();
            if (v == "Biodiversity")
                r.rep_biodiversity = true;
            else if (v == "Counter")
                r.rep_counter = true;
            else if (v == "Execution")
                r.rep_execution = true;
            else if (v == "Csv")
                r.csv_output = need(*n, "output").text;
            else if (v == "GlobalSpeciation")
                r.speciation_output = need(*n, "output").text;
            else if (v == "GlobalTurnover")
                r.turnover_output = need(*n, "output").text;
            else if (v == "GlobalCoverage")
                r.coverage_output = need(*n, "output").text;
            else
                std::fprintf(stderr, "necsim-b200: reporter %s is not provided here and is ignored\n", v.c_str());
        }
    }
}

// the configuration with the remaining lineages as a List sample in Resume
// mode and no pause (rustcoalescence/src/cli/simulate/pause.rs:20-60)
// (pause.rs:20-61: mode Resume, or Restart(after: the pause time) for the
// Restart pause mode)
std::string resume_config(const std::string &text, uint64_t seed, const std::vector<necsim_lineage> &rem,
                          bool restart, double after, const std::string &bincode_file, LineageFileSaver *saver) {
    Value root = necsim::ron::parse(text);
    Value sample;
    sample.kind = Value::Struct;
    sample.text = "Sample";
    Value pct;
    pct.kind = Value::Number;
    pct.text = "1.0";
    sample.fields.emplace_back("percentage", pct);
    Value origin;
    origin.kind = Value::Struct;
    origin.text = "List";
    Value list;
    list.kind = Value::List;
    char buf[64];
    for (const necsim_lineage &l : rem) {
        Value lin;
        lin.kind = Value::Struct;
        lin.text = "Lineage";
        Value ref, time, loc;
        ref.kind = Value::Number;
        ref.text = std::to_string(l.global_reference);
        time.kind = Value::Number;
        std::snprintf(buf, sizeof(buf), "%.17g", l.last_event_time);
        time.text = buf;
        if (time.text.find_first_of(".eEn") == std::string::npos) time.text += ".0";
        loc.kind = Value::Struct;
        for (auto kv : {std::make_pair("x", l.x), std::make_pair("y", l.y), std::make_pair("i", l.index)}) {
            Value c;
            c.kind = Value::Number;
            c.text = std::to_string(kv.second);
            loc.fields.emplace_back(kv.first, c);
        }
        lin.fields.emplace_back("ref", ref);
        lin.fields.emplace_back("time", time);
        lin.fields.emplace_back("loc", loc);
        list.items.push_back(lin);
    }
    origin.items.push_back(list);
    if (!bincode_file.empty()) {
        // destiny Bincode(file) (pause.rs:29-39): the lineages go to the file
        // created when the configuration was read
        if (!saver) fail("no lineage file was created for " + bincode_file);
        saver->write(rem);
        origin = Value{};
        origin.kind = Value::Struct;
        origin.text = "Bincode";
        Value file;
        file.kind = Value::String;
        file.text = bincode_file;
        origin.fields.emplace_back("file", file);
    }
    sample.fields.emplace_back("origin", origin);
    Value mode;
    mode.kind = Value::Ident;
    mode.text = "Resume";
    if (restart) {
        mode.kind = Value::Struct;
        mode.text = "Restart";
        Value a;
        a.kind = Value::Number;
        std::snprintf(buf, sizeof(buf), "%.17g", after);
        a.text = buf;
        if (a.text.find_first_of(".eEn") == std::string::npos) a.text += ".0";
        mode.fields.emplace_back("after", a);
    }
    sample.fields.emplace_back("mode", mode);
    Value none;
    none.kind = Value::Ident;
    none.text = "None";
    Value rng;
    rng.kind = Value::Struct;
    rng.text = "Seed";
    Value sv;
    sv.kind = Value::Number;
    sv.text = std::to_string(seed);
    rng.items.push_back(sv);
    bool has_sample = false, has_pause = false, has_rng = false;
    for (auto &f : root.fields) {
        if (f.first == "sample") f.second = sample, has_sample = true;
        if (f.first == "pause") f.second = none, has_pause = true;
        if (f.first == "rng") f.second = rng, has_rng = true;
    }
    if (!has_sample) root.fields.emplace_back("sample", sample);
    if (!has_pause) root.fields.emplace_back("pause", none);
    if (!has_rng) root.fields.emplace_back("rng", rng);
    return necsim::ron::to_string(root) + "\n";
}

// The Counter reporter (necsim/plugins/common/src/event_counter.rs): it
// collapses an event equal to the one before it (speciation: origin and time;
// dispersal: origin, time and target) and counts such a repeat as a late
// coalescence when its prior time differs from the last one seen.  Every
// dispersal here carries LineageInteraction::Maybe, the Independent
// coalescence sampler's (coalescence_sampler/independent.rs:52), so every
// deduplicated dispersal is "detected late".
struct EventCounter {
    uint64_t raw_total = 0, speciation = 0, self_dispersal = 0, out_dispersal = 0, self_coalescence = 0,
             out_coalescence = 0, late_dispersal_coalescence = 0, late_coalescence = 0;
    bool has_spec = false, has_disp = false, has_prior = false;
    necsim_speciation_event last_spec{};
    necsim_dispersal_event last_disp{};
    double last_prior = 0.0;

    void repeat(double prior) {
        if (!has_prior || prior != last_prior) late_coalescence += 1;
        last_prior = prior;
        has_prior = true;
    }
    void on(const necsim_speciation_event &e) {
        raw_total += 1;
        if (has_spec && e.x == last_spec.x && e.y == last_spec.y && e.index == last_spec.index &&
            e.event_time == last_spec.event_time)
            return repeat(e.prior_time);
        last_spec = e;
        has_spec = true;
        last_prior = e.prior_time;
        has_prior = true;
        speciation += 1;
    }
    void on(const necsim_dispersal_event &e) {
        raw_total += 1;
        if (has_disp && e.x == last_disp.x && e.y == last_disp.y && e.index == last_disp.index &&
            e.event_time == last_disp.event_time && e.target_x == last_disp.target_x &&
            e.target_y == last_disp.target_y && e.target_index == last_disp.target_index)
            return repeat(e.prior_time);
        last_disp = e;
        has_disp = true;
        last_prior = e.prior_time;
        has_prior = true;
        late_dispersal_coalescence += 1;  // LineageInteraction::Maybe
    }
    // event_counter.rs finalise: the summary, when any event was seen
    void print() const {
        if (!has_spec && !has_disp) return;
        std::printf("Event Summary:\n - Total #individuals:\n   %" PRIu64 "\n",
                    speciation + self_coalescence + out_coalescence + late_coalescence);
        std::printf(" - Total #events:\n   - raw:\n     %" PRIu64 "\n   - deduplicated:\n     %" PRIu64 "\n",
                    raw_total,
                    speciation + self_coalescence + out_coalescence + self_dispersal + out_dispersal +
                        late_dispersal_coalescence);
        std::printf(" - Speciation:\n    %" PRIu64 "\n", speciation);
        std::printf(" - Dispersal:\n   - same location, no coalescence:\n     %" PRIu64
                    "\n   - same location, with coalescence:\n     %" PRIu64
                    "\n   - new location, no coalescence:\n     %" PRIu64
                    "\n   - new location, with coalescence:\n     %" PRIu64
                    "\n   - detected late, no coalescence:\n     %" PRIu64
                    "\n   - detected late, with coalescence:\n     %" PRIu64 "\n",
                    self_dispersal, self_coalescence, out_dispersal, out_coalescence,
                    late_dispersal_coalescence - late_coalescence,  // usize arithmetic, wrapping in release
                    late_coalescence);
    }
};

// Rust's Display for a finite f64: the shortest round-trip digits
// (std::to_chars' scientific form), written out in fixed notation with zeros
// filling any place beyond them (2^60 prints as 1152921504606847000)
std::string rust_f64_display(double v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char t[64];
    const auto end = std::to_chars(t, t + sizeof(t), v, std::chars_format::scientific).ptr;
    std::string sci(t, end), out;
    if (!sci.empty() && sci[0] == '-') {
        out = "-";
        sci.erase(0, 1);
    }
    const size_t e = sci.find('e');
    std::string digits = sci.substr(0, e);
    digits.erase(std::remove(digits.begin(), digits.end(), '.'), digits.end());
    const long x = std::strtol(sci.c_str() + e + 1, nullptr, 10);  // value = d1.d2.. * 10^x
    const long n = (long)digits.size();
    if (x >= n - 1) {
        out += digits + std::string((size_t)(x - (n - 1)), '0');
    } else if (x >= 0) {
        out += digits.substr(0, (size_t)x + 1) + "." + digits.substr((size_t)x + 1);
    } else {
        out += "0." + std::string((size_t)(-x - 1), '0') + digits;
    }
    return out;
}

// A reporter's output file: created and truncated, with its header line.
FILE *open_output(const std::string &path, const char *header) {
    if (path.empty()) return nullptr;
    FILE *f = std::fopen(path.c_str(), "w");  // initialise(): create + truncate
    if (!f) fail("cannot write the reporter output " + path);
    std::fprintf(f, "%s\n", header);
    return f;
}

// The statistics plugin (necsim/plugins/statistics/src/{speciation,turnover,
// coverage}.rs): GlobalSpeciation writes each speciation's event time,
// GlobalTurnover the time since the lineage's previous event for every
// speciation and dispersal, GlobalCoverage each dispersal's origin and
// target.  Each skips an event equal to the previous one of its kind
// (event.rs:299-318: the same origin and event time, and target).
struct StatisticsWriters {
    FILE *speciation = nullptr, *turnover = nullptr, *coverage = nullptr;
    bool have_spec = false, have_disp = false;
    necsim_speciation_event last_spec{};
    necsim_dispersal_event last_disp{};
    explicit StatisticsWriters(const Run &r)
        : speciation(open_output(r.speciation_output, "speciation")),
          turnover(open_output(r.turnover_output, "turnover")),
          coverage(open_output(r.coverage_output, "x-from,y-from,index-from,x-to,y-to,index-to")) {}
    ~StatisticsWriters() {
        for (FILE *f : {speciation, turnover, coverage})
            if (f) std::fclose(f);
    }
    StatisticsWriters(const StatisticsWriters &) = delete;
    StatisticsWriters &operator=(const StatisticsWriters &) = delete;
    void on(const necsim_speciation_event *ev, uint64_t n) {
        for (uint64_t i = 0; i < n; ++i) {
            const necsim_speciation_event &e = ev[i];
            if (have_spec && e.x == last_spec.x && e.y == last_spec.y && e.index == last_spec.index &&
                e.event_time == last_spec.event_time)
                continue;
            have_spec = true;
            last_spec = e;
            if (speciation) std::fprintf(speciation, "%s\n", rust_f64_display(e.event_time).c_str());
            if (turnover) std::fprintf(turnover, "%s\n", rust_f64_display(e.event_time - e.prior_time).c_str());
        }
    }
    void on(const necsim_dispersal_event *ev, uint64_t n) {
        for (uint64_t i = 0; i < n; ++i) {
            const necsim_dispersal_event &e = ev[i];
            if (have_disp && e.x == last_disp.x && e.y == last_disp.y && e.index == last_disp.index &&
                e.event_time == last_disp.event_time && e.target_x == last_disp.target_x &&
                e.target_y == last_disp.target_y && e.target_index == last_disp.target_index)
                continue;
            have_disp = true;
            last_disp = e;
            if (turnover) std::fprintf(turnover, "%s\n", rust_f64_display(e.event_time - e.prior_time).c_str());
            if (coverage)
                std::fprintf(coverage, "%u,%u,%u,%u,%u,%u\n", e.x, e.y, e.index, e.target_x, e.target_y,
                             e.target_index);
        }
    }
};

// The Csv reporter (necsim/plugins/csv/src/lib.rs): the header, then one
// line per event in delivery order, `reference,time,x,y,index,type` with the
// event's origin and type 's' (speciation) or 'd' (dispersal).  Times print
// as Rust's Display for f64 does: the shortest digits that read back to the
// same value, without an exponent.
struct CsvWriter {
    FILE *f = nullptr;
    explicit CsvWriter(const std::string &path) : f(open_output(path, "reference,time,x,y,index,type")) {}
    ~CsvWriter() {
        if (f) std::fclose(f);
    }
    CsvWriter(const CsvWriter &) = delete;
    CsvWriter &operator=(const CsvWriter &) = delete;
    void row(uint64_t gref, double time, uint32_t x, uint32_t y, uint32_t index, char type) {
        if (!f) return;
        std::fprintf(f, "%" PRIu64 ",%s,%u,%u,%u,%c\n", gref, rust_f64_display(time).c_str(), x, y, index, type);
    }
    void speciation(const necsim_speciation_event *ev, uint64_t n) {
        for (uint64_t i = 0; f && i < n; ++i)
            row(ev[i].global_lineage_reference, ev[i].event_time, ev[i].x, ev[i].y, ev[i].index, 's');
    }
    void dispersal(const necsim_dispersal_event *ev, uint64_t n) {
        for (uint64_t i = 0; f && i < n; ++i)
            row(ev[i].global_lineage_reference, ev[i].event_time, ev[i].x, ev[i].y, ev[i].index, 'd');
    }
};

struct Counts {
    EventCounter counter;
    necsim_reporter log{};  // the event log's reporter, when one is written
    CsvWriter *csv = nullptr;
    StatisticsWriters *stats = nullptr;
};

int on_speciation(void *user, const necsim_speciation_event *ev, uint64_t n) {
    Counts &c = *static_cast<Counts *>(user);
    for (uint64_t i = 0; i < n; ++i) c.counter.on(ev[i]);
    if (c.csv) c.csv->speciation(ev, n);
    if (c.stats) c.stats->on(ev, n);
    if (c.log.report_speciation) return c.log.report_speciation(c.log.user, ev, n);
    return 0;
}

int on_dispersal(void *user, const necsim_dispersal_event *ev, uint64_t n) {
    Counts &c = *static_cast<Counts *>(user);
    if (c.log.report_dispersal && c.log.report_dispersal(c.log.user, ev, n) != 0) return 1;
    for (uint64_t i = 0; i < n; ++i) c.counter.on(ev[i]);
    if (c.csv) c.csv->dispersal(ev, n);
    if (c.stats) c.stats->on(ev, n);
    return 0;
}

// A duration as Rust's `Debug for Duration` prints it (the Execution
// reporter's `{:?}`, plugins/common/src/execution_time.rs:65-76): the
// largest unit among s, ms, µs and ns with at least one whole unit, then the
// fraction's significant digits
template <typename D>
std::string rust_duration(D d) {
    const uint64_t ns = (uint64_t)std::max<int64_t>(0, std::chrono::duration_cast<std::chrono::nanoseconds>(d).count());
    uint64_t unit = 1;
    const char *name = "ns";
    int digits = 0;
    if (ns >= 1000000000ULL) {
        unit = 1000000000ULL, name = "s", digits = 9;
    } else if (ns >= 1000000ULL) {
        unit = 1000000ULL, name = "ms", digits = 6;
    } else if (ns >= 1000ULL) {
        unit = 1000ULL, name = "\u00b5s", digits = 3;
    }
    std::string out = std::to_string(ns / unit);
    uint64_t frac = ns % unit;
    if (frac) {
        std::string f = std::to_string(frac);
        f.insert(0, (size_t)digits - f.size(), '0');
        while (!f.empty() && f.back() == '0') f.pop_back();
        out += "." + f;
    }
    return out + name;
}

std::string slurp(const std::string &path) {
    std::ifstream f(path);
    if (!f) fail("cannot read " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

int simulate(const std::string &path, bool run) {
    const std::string text = slurp(path);
    Run r = parse_config(text);
    if (r.entropy) {
        std::random_device rd;
        r.seed = ((uint64_t)rd() << 32) ^ rd();
    }
    // the origins to simulate
    std::vector<necsim_lineage> lineages;
    if (!r.resume) {
        uint64_t n = 0;
        int rc = necsim_enumerate_origins(&r.sc, nullptr, 0, &n);
        if (rc) fail("invalid scenario (status " + std::to_string(rc) + ")");
        std::vector<necsim_lineage> all(n);
        rc = necsim_enumerate_origins(&r.sc, all.data(), n, &n);
        if (rc) fail("origin enumeration failed (status " + std::to_string(rc) + ")");
        // IsolatedLandscape samples every origin, then keeps its subdomain's
        // (independent/src/launch.rs:101-110, origin_sampler/decomposition.rs)
        const uint32_t prank = r.landscape ? 0 : r.rank, psize = r.landscape ? 1 : r.size;
        uint64_t k = 0;
        necsim_presample_origins(n, r.percentage, prank, psize, nullptr, 0, &k);
        std::vector<uint64_t> pos(k);
        rc = necsim_presample_origins(n, r.percentage, prank, psize, pos.data(), k, &k);
        if (rc) fail("invalid sample percentage or partition");
        lineages.reserve(k);
        for (uint64_t p : pos) lineages.push_back(all[p]);
    } else if (!r.landscape) {
        // a resumed sample is partitioned like fresh origins
        for (size_t j = r.rank; j < r.list.size(); j += r.size) lineages.push_back(r.list[j]);
    } else {
        lineages = r.list;
    }
    if (r.landscape) {
        std::vector<uint32_t> ranks(lineages.size());
        int32_t exact = 1;
        const int rc = necsim_subdomain_ranks(&r.sc, r.size, lineages.data(), lineages.size(), ranks.data(), &exact);
        if (rc) fail("landscape decomposition failed (status " + std::to_string(rc) + ")");
        if (!exact)
            std::fprintf(stderr, "necsim-b200: warning: the habitat could not be partitioned into %u partition(s)\n",
                         r.size);
        size_t m = 0;
        for (size_t j = 0; j < lineages.size(); ++j)
            if (ranks[j] == r.rank) lineages[m++] = lineages[j];
        lineages.resize(m);
    }
    std::printf("necsim-b200: %s, speciation %g, seed %" PRIu64 ", %zu lineages%s\n", r.summary.c_str(),
                r.speciation, r.seed, lineages.size(), r.restart ? " (restarted)" : (r.resume ? " (resumed)" : ""));
    if (r.restart) std::printf("necsim-b200: restart after t = %.17g\n", r.restart_after);
    std::printf("necsim-b200: algorithm %s, %s event times, delta_t %g, step_slice %" PRIu64 "\n",
                r.algorithm.c_str(), r.args.event_time_sampler == NECSIM_SAMPLER_EXP ? "exponential" : "Poisson",
                r.args.delta_t > 0.0 ? r.args.delta_t : 2.0, r.args.step_slice ? r.args.step_slice : (uint64_t)10);
    if (r.pause_before >= 0.0) std::printf("necsim-b200: pause before t = %g -> %s\n", r.pause_before,
                                           r.pause_config.c_str());
    if (!run) return 0;

    const auto t0 = std::chrono::steady_clock::now();
    necsim_ctx *ctx = nullptr;
    int rc = necsim_gpu_create(&r.sc, &r.args, &ctx);
    if (rc) {
        const std::string m = ctx ? necsim_gpu_last_error(ctx) : "";
        necsim_gpu_destroy(ctx);
        fail("set-up failed (status " + std::to_string(rc) + "): " + m);
    }
    Counts counts;
    CsvWriter csv(r.csv_output);
    counts.csv = &csv;
    StatisticsWriters stats(r);
    counts.stats = &stats;
    necsim_event_log *log = nullptr;
    if (!r.log_directory.empty()) {
        rc = necsim_event_log_create(r.log_directory.c_str(), r.log_capacity, 1, r.args.report_dispersal, &log);
        if (rc) {
            necsim_gpu_destroy(ctx);
            fail("cannot create the event log " + r.log_directory + " (start from a clean log directory)");
        }
        counts.log = necsim_event_log_reporter(log);
    }
    necsim_reporter rep{&counts, on_speciation, on_dispersal};
    necsim_outcome out{};
    const auto t1 = std::chrono::steady_clock::now();
    rc = necsim_gpu_simulate_lineages(ctx, lineages.data(), lineages.size(), r.restart_after, necsim_seed_from_u64(r.seed),
                                      r.pause_before, &rep, &out);
    const auto t2 = std::chrono::steady_clock::now();
    if (rc) {
        const std::string m = necsim_gpu_last_error(ctx);
        necsim_gpu_destroy(ctx);
        fail("simulation failed (status " + std::to_string(rc) + "): " + m);
    }
    std::vector<necsim_lineage> rem;
    if (out.paused) {
        uint64_t n = out.n_remaining;
        rem.resize(n);
        rc = necsim_gpu_remaining_lineages(ctx, rem.data(), n, &n);
        if (rc) fail("could not read the remaining lineages");
    }
    necsim_gpu_destroy(ctx);
    if (log && necsim_event_log_close(log) != 0) fail("could not write the event log");
    if (log) std::printf("necsim-b200: events logged to %s\n", r.log_directory.c_str());
    const auto t3 = std::chrono::steady_clock::now();

    std::printf("necsim-b200: %s after %" PRIu64 " steps at time %.17g\n", out.paused ? "paused" : "done",
                out.steps, out.time);
    if (r.rep_biodiversity && out.biodiversity > 0)
        std::printf("The simulation resulted in a biodiversity of %" PRIu64 " unique species.\n",
                    out.biodiversity);
    if (r.rep_counter) counts.counter.print();
    if (r.rep_execution) {
        std::printf("The simulation took:\n - initialisation: %s\n - execution: %s\n - cleanup: %s\n",
                    rust_duration(t1 - t0).c_str(), rust_duration(t2 - t1).c_str(), rust_duration(t3 - t2).c_str());
    }
    if (out.paused && !r.pause_config.empty()) {
        std::ofstream f(r.pause_config);
        if (!f) fail("cannot write " + r.pause_config);
        f << resume_config(text, r.seed, rem, r.pause_restart, r.pause_before, r.pause_bincode, r.pause_saver.get());
        std::printf("necsim-b200: %zu remaining lineages written to %s\n", rem.size(), r.pause_config.c_str());
    }
    return 0;
}

// ---- replay (rustcoalescence/src/cli/replay.rs, args/cli/replay.rs) ----

// The reporters of a replay: Biodiversity counts speciation events that
// differ from the previous one by origin or event time (biodiversity.rs:33-41),
// Counter as in a simulation.
struct ReplayCounts {
    uint64_t biodiversity = 0;
    bool have_last = false;
    necsim_speciation_event last{};
    EventCounter counter;
    CsvWriter *csv = nullptr;
    StatisticsWriters *stats = nullptr;
};

int replay_speciation(void *user, const necsim_speciation_event *ev, uint64_t n) {
    ReplayCounts &c = *static_cast<ReplayCounts *>(user);
    if (c.csv) c.csv->speciation(ev, n);
    if (c.stats) c.stats->on(ev, n);
    for (uint64_t i = 0; i < n; ++i) {
        c.counter.on(ev[i]);
        const necsim_speciation_event &e = ev[i];
        if (c.have_last && e.x == c.last.x && e.y == c.last.y && e.index == c.last.index &&
            e.event_time == c.last.event_time)
            continue;
        c.last = e;
        c.have_last = true;
        c.biodiversity += 1;
    }
    return 0;
}

int replay_dispersal(void *user, const necsim_dispersal_event *ev, uint64_t n) {
    ReplayCounts &c = *static_cast<ReplayCounts *>(user);
    for (uint64_t i = 0; i < n; ++i) c.counter.on(ev[i]);
    if (c.csv) c.csv->dispersal(ev, n);
    if (c.stats) c.stats->on(ev, n);
    return 0;
}

// the segment files a pattern names (replay/globbed.rs): its matches in
// order, files only when several match, or the pattern itself when nothing
// matches
std::vector<std::string> expand_segments(const std::string &pattern) {
    std::vector<std::string> out;
    glob_t g;
    std::memset(&g, 0, sizeof(g));
    const int rc = glob(pattern.c_str(), 0, nullptr, &g);
    if (rc == 0 && g.gl_pathc == 1) {
        out.push_back(g.gl_pathv[0]);
    } else if (rc == 0) {
        for (size_t i = 0; i < g.gl_pathc; ++i) {
            struct stat st;
            if (stat(g.gl_pathv[i], &st) != 0 || S_ISREG(st.st_mode)) out.push_back(g.gl_pathv[i]);
        }
    } else {
        out.push_back(pattern);
    }
    globfree(&g);
    return out;
}

int replay(const std::string &path) {
    const Value root = necsim::ron::parse(slurp(path));
    const Value *log = root.field("log") ? root.field("log") : root.field("event_log");
    if (!log) fail("missing field `log`");
    std::vector<std::string> segs;
    for (const Value &p : need(*log, "segments").items)
        for (const std::string &s : expand_segments(p.text)) segs.push_back(s);
    uint64_t capacity = 100000;  // default_event_log_replay_segment_capacity
    if (const Value *c = log->field("capacity")) capacity = c->as_u64();
    bool strict = true;
    if (const Value *m = root.field("mode")) {
        if (m->variant() == "WarnOnly") strict = false;
        else if (m->variant() != "Strict") fail("replay mode must be Strict or WarnOnly");
    }
    Run r;
    parse_reporters(root, r);
    std::printf("necsim-b200: replaying %zu event log segment(s)\n", segs.size());
    std::vector<const char *> ptrs;
    for (const std::string &s : segs) ptrs.push_back(s.c_str());
    ReplayCounts counts;
    CsvWriter csv(r.csv_output);
    counts.csv = &csv;
    StatisticsWriters stats(r);
    counts.stats = &stats;
    necsim_reporter rep{&counts, replay_speciation, replay_dispersal};
    char err[512];
    uint64_t n = 0;
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = necsim_event_log_replay(ptrs.data(), ptrs.size(), capacity, r.needs_speciation() ? 1 : 0,
                                           r.needs_dispersal() ? 1 : 0, strict ? 1 : 0, &rep, &n, err, sizeof(err));
    const auto t1 = std::chrono::steady_clock::now();
    if (rc) fail(std::string("replay failed: ") + err);
    if (err[0]) std::fprintf(stderr, "necsim-b200: warning: %s\n", err);
    std::printf("necsim-b200: replayed %" PRIu64 " events\n", n);
    if (r.rep_biodiversity && counts.biodiversity > 0)
        std::printf("The simulation resulted in a biodiversity of %" PRIu64 " unique species.\n", counts.biodiversity);
    if (r.rep_counter) counts.counter.print();
    if (r.rep_execution)
        std::printf("The replay took %s\n", rust_duration(t1 - t0).c_str());
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    const bool known = argc == 3 && (std::strcmp(argv[1], "simulate") == 0 || std::strcmp(argv[1], "check") == 0 ||
                                      std::strcmp(argv[1], "replay") == 0);
    if (!known) {
        std::fprintf(stderr, "usage: necsim-b200 simulate|check|replay <config.ron>\n");
        return 2;
    }
    try {
        if (std::strcmp(argv[1], "replay") == 0) return replay(argv[2]);
        return simulate(argv[2], std::strcmp(argv[1], "simulate") == 0);
    } catch (const Fail &f) {
        std::fprintf(stderr, "necsim-b200: %s\n", f.msg.c_str());
    } catch (const necsim::ron::ParseError &e) {
        std::fprintf(stderr, "necsim-b200: configuration error (line %zu): %s\n", e.line, e.msg.c_str());
    } catch (const std::exception &e) {
        std::fprintf(stderr, "necsim-b200: %s\n", e.what());
    }
    return 1;
}
