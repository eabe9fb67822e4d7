// tables.cpp -- SpatiallyExplicit dispersal tables, built row-parallel on
// the host.  The per-row arithmetic follows the reference's construction
// step for step (weights, left-fold sums, Vose's stack order, the
// self-dispersal atom moved last) because the GPU's draws index these
// tables directly and must land on the same atoms as the reference.
#include "tables.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>

namespace necsim {

namespace {

struct RowScratch {
    std::vector<uint32_t> ev;
    std::vector<double> w;
    std::vector<uint32_t> over, under;
};

// alias/packed.rs:59-121 AliasMethodSamplerAtom::create into `out`
void vose(const uint32_t *ev, const double *w, size_t n, AliasAtom *out, RowScratch &s) {
    double total = 0.0;
    for (size_t i = 0; i < n; ++i) total = total + w[i];  // Sum: left fold from 0
    const double nf = (double)n;
    for (size_t i = 0; i < n; ++i) {
        out[i].u = w[i] * nf / total;
        out[i].e = ev[i];
        out[i].k = ev[i];
    }
    s.over.clear();
    s.under.clear();
    for (size_t i = 0; i < n; ++i)
        if (out[i].u > 1.0) s.over.push_back((uint32_t)i);
    for (size_t i = 0; i < n; ++i)
        if (out[i].u < 1.0) s.under.push_back((uint32_t)i);
    while (!s.over.empty() && !s.under.empty()) {
        const uint32_t o = s.over.back();
        s.over.pop_back();
        const uint32_t u = s.under.back();
        s.under.pop_back();
        out[o].u = out[o].u + out[u].u - 1.0;
        out[u].k = out[o].e;
        if (out[o].u < 1.0)
            s.under.push_back(o);
        else if (out[o].u > 1.0)
            s.over.push_back(o);
    }
    for (uint32_t i : s.over) out[i].u = 1.0;
    for (uint32_t i : s.under) out[i].u = 1.0;
}

// Collects row `r`'s positive weights p(r, c) * habitat(c) in column order.
void row_weights(const necsim_scenario &sc, uint64_t r, RowScratch &s, double &self_w) {
    const uint64_t n = (uint64_t)sc.width * sc.height;
    const double *row = sc.dispersal + r * n;
    s.ev.clear();
    s.w.clear();
    self_w = 0.0;
    for (uint64_t c = 0; c < n; ++c) {
        const double weight = row[c] * (double)sc.habitat[c];
        if (weight > 0.0) {
            s.ev.push_back((uint32_t)c);
            s.w.push_back(weight);
            if (c == r) self_w = weight;
        }
    }
}

template <typename F>
void parallel_rows(uint64_t n, unsigned threads, F &&f) {
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    threads = (unsigned)std::min<uint64_t>(threads, std::max<uint64_t>(1, n / 64));
    if (threads <= 1) {
        RowScratch s;
        for (uint64_t r = 0; r < n; ++r) f(r, s);
        return;
    }
    std::atomic<uint64_t> next{0};
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < threads; ++t)
        pool.emplace_back([&] {
            RowScratch s;
            for (;;) {
                const uint64_t r0 = next.fetch_add(64);
                if (r0 >= n) break;
                const uint64_t r1 = std::min(n, r0 + 64);
                for (uint64_t r = r0; r < r1; ++r) f(r, s);
            }
        });
    for (auto &t : pool) t.join();
}

}  // namespace

bool dispersal_contract_holds(const necsim_scenario &sc) {
    const uint64_t n = (uint64_t)sc.width * sc.height;
    std::atomic<bool> ok{true};
    parallel_rows(n, 0, [&](uint64_t r, RowScratch &) {
        if (!ok.load(std::memory_order_relaxed)) return;
        const double *row = sc.dispersal + r * n;
        if (sc.habitat[r] > 0) {
            bool any = false;
            for (uint64_t c = 0; c < n; ++c) {
                if (row[c] > 0.0) {
                    if (sc.habitat[c] == 0) {
                        ok = false;
                        return;
                    }
                    any = true;
                }
            }
            if (!any) ok = false;
        } else {
            for (uint64_t c = 0; c < n; ++c)
                if (row[c] != 0.0) {
                    ok = false;
                    return;
                }
        }
    });
    return ok.load();
}

float dispersal_entropy(const necsim_scenario &sc, uint64_t r) {
    if (!sc.dispersal) return 0.0f;
    RowScratch s;
    double self_w;
    row_weights(sc, r, s, self_w);
    if (s.ev.empty()) return 0.0f;
    double total = 0.0;
    for (double w : s.w) total = total + w;
    double h = 0.0;
    for (double w : s.w) {
        const double q = w / total;
        h -= q * std::log(q);
    }
    return (float)h;
}

int build_spatially_explicit_tables(const necsim_scenario &sc, HostTables &out, unsigned threads) {
    const uint64_t n = (uint64_t)sc.width * sc.height;
    out.cells.assign(n, CellRecord{});
    // injection prefix sums (habitat/in_memory.rs:143-163)
    uint64_t acc = 0;
    for (uint64_t c = 0; c < n; ++c) {
        out.cells[c].injection = acc;
        out.cells[c].habitat = sc.habitat[c];
        acc += sc.habitat[c];
    }
    if (acc == 0) return 1;
    if (!dispersal_contract_holds(sc)) return 2;

    // pass 1: atoms per row (self-dispersal leaves the atoms when its
    // bucket would be over-full, mod.rs:141-174)
    std::vector<uint64_t> count(n, 0);
    std::vector<double> sd_prob(n, 0.0);
    std::vector<uint8_t> sd_separate(n, 0);
    out.entropy.assign(n, 0.0f);
    parallel_rows(n, threads, [&](uint64_t r, RowScratch &s) {
        double self_w;
        row_weights(sc, r, s, self_w);
        if (s.ev.empty()) return;
        double total = 0.0;
        for (double w : s.w) total = total + w;
        double h = 0.0;
        for (double w : s.w) {
            const double q = w / total;
            h -= q * std::log(q);
        }
        out.entropy[r] = (float)h;
        sd_prob[r] = self_w / total;
        const double sd_u = self_w * (double)s.ev.size() / total;
        if (sd_u < 1.0) {
            count[r] = s.ev.size();
        } else {
            sd_separate[r] = 1;
            count[r] = s.ev.size() - 1;
        }
    });
    uint64_t total_atoms = 0;
    for (uint64_t r = 0; r < n; ++r) {
        out.cells[r].atom_start = (uint32_t)total_atoms;
        out.cells[r].atom_count = (uint32_t)count[r];
        total_atoms += count[r];
        if (total_atoms > 0xffffffffULL) return 3;
    }
    out.atoms.assign(total_atoms, AliasAtom{});

    // pass 2: build each row's atoms in place
    parallel_rows(n, threads, [&](uint64_t r, RowScratch &s) {
        CellRecord &rec = out.cells[r];
        rec.self_dispersal = 0.0;
        rec.non_self_event = (uint32_t)r;
        double self_w;
        row_weights(sc, r, s, self_w);
        if (s.ev.empty()) return;
        rec.self_dispersal = sd_prob[r];
        AliasAtom *atoms = out.atoms.data() + rec.atom_start;
        if (!sd_separate[r]) {
            const size_t m = s.ev.size();
            vose(s.ev.data(), s.w.data(), m, atoms, s);
            // the atom holding self-dispersal goes last, self-dispersal in k
            for (size_t i = 0; i < m; ++i) {
                if (atoms[i].e == (uint32_t)r || atoms[i].k == (uint32_t)r) {
                    if (atoms[i].e == (uint32_t)r) {
                        std::swap(atoms[i].e, atoms[i].k);
                        atoms[i].u = 1.0 - atoms[i].u;
                    }
                    rec.non_self_event = atoms[i].e;
                    std::swap(atoms[i], atoms[m - 1]);
                    break;
                }
            }
        } else {
            size_t m = 0;
            for (size_t i = 0; i < s.ev.size(); ++i)
                if (s.ev[i] != (uint32_t)r) {
                    s.ev[m] = s.ev[i];
                    s.w[m] = s.w[i];
                    ++m;
                }
            vose(s.ev.data(), s.w.data(), m, atoms, s);
        }
    });
    return 0;
}

}  // namespace necsim
