// Host-side check of two shared-memory layouts, compiled by nvcc and run on
// the CPU (no GPU is involved): the multi-pass kernel's exchange (pass_xidx in
// zlfft_pass.cuh), and the macro path's segment tiles (TileWorker::keep_idx in
// zlfft_tile.cuh, the columns kept for the transposed store).
//
// For every pass whose unit rows are shorter than a 128-byte line (the 512-
// and 1024-point passes, XOR-swizzled layout), it replays the positions each
// shared-memory access of pass_kernel touches (the group reads, the exchange
// writes, the first pass's staging writes and column-wise copy-out) through
// the kernel's own index function, and checks that
//   - the layout is a bijection of (position, unit slot) onto the buffer;
//   - every access is free of bank conflicts: within each phase of the warp
//     (16 lanes for 8-byte elements, 8 for 16-byte ones), no two lanes touch
//     different addresses in the same bank group of a 128-byte line.
// Exit status 0 when every configuration passes; the failures are printed.
#include <cstdio>
#include <map>
#include <set>
#include <vector>

#include "zlfft_macro.cuh"
#include "zlfft_pass.cuh"

using namespace zlfft;

namespace {

int g_fail = 0;
bool g_quiet = false;  // the control run: its failures are expected, not printed

// Wavefronts above one per phase: phase lanes that share a bank group but not an address.
template <class Cfg>
int conflicts(const std::vector<int>& idx) {
    using C = typename Cfg::C;
    const int lanes = 128 / (int)sizeof(C);  // lanes per phase
    int extra = 0;
    for (size_t ph = 0; ph < idx.size(); ph += lanes) {
        std::map<int, std::set<int>> bank;  // bank group -> element indices
        for (size_t l = ph; l < ph + lanes && l < idx.size(); ++l) bank[idx[l] % Cfg::SLOTS].insert(idx[l]);
        int worst = 1;
        for (auto& kv : bank) worst = (int)kv.second.size() > worst ? (int)kv.second.size() : worst;
        extra += worst - 1;
    }
    return extra;
}

// One warp-wide access: pos(t) and unit(t) for the 32 lanes of warp w.
template <class Cfg, class PosFn, class UnitFn>
void access(const char* what, int w, PosFn pt_pc, UnitFn unit, int& total) {
    std::vector<int> idx;
    for (int lane = 0; lane < 32; ++lane) {
        const int t = 32 * w + lane;
        if (t >= Cfg::THREADS) break;
        int pt, pc;
        pt_pc(t, pt, pc);
        idx.push_back(pass_xidx<Cfg>(pt, pc, unit(t)));
    }
    const int c = conflicts<Cfg>(idx);
    if (c && total == 0 && !g_quiet) std::printf("  first conflict: %s, warp %d, %d extra wavefronts\n", what, w, c);
    total += c;
}

// Replays the pass's accesses through pass_xidx<Cfg>; returns the extra
// wavefronts (0: conflict-free) and counts layout errors in *bad.
template <class Cfg, int P, int S>
int replay(int* bad_out) {
    constexpr int R = Cfg::R, E = Cfg::E, T = Cfg::T, UPC = Cfg::UPC, L_IN = Cfg::L_IN;
    int bad = 0;
    // bijection onto [0, R * UPC)
    std::set<int> seen;
    for (int pos = 0; pos < R; ++pos)
        for (int u = 0; u < UPC; ++u) {
            const int i = pass_xidx<Cfg>(pos, 0, u);
            if (i < 0 || i >= R * UPC || !seen.insert(i).second) ++bad;
        }
    if (bad && !g_quiet) std::printf("  %d slots out of range or taken twice\n", bad);
    // a split into disjoint parts gives the position's own index
    for (int pt = 0; pt < R; ++pt)
        for (int pc = 0; pc < R; pc += 1)
            if ((pt & pc) == 0 && pt + pc < R)
                for (int u = 0; u < UPC; ++u)
                    if (pass_xidx<Cfg>(pt, pc, u) != pass_xidx<Cfg>(pt + pc, 0, u)) ++bad;
    if (bad && !g_quiet) std::printf("  a disjoint split changes the index\n");
    int total = 0;
    auto unit = [](int t) { return t % UPC; };
    for (int g = Cfg::GB; g < Cfg::GE; ++g) {
        const Grp G = pass_group(P, S, g);
        const int NB = E / G.R, ELL = G.L / L_IN, GI = g - Cfg::GB;
        const bool last = g + 1 == Cfg::GE;
        for (int w = 0; w < Cfg::THREADS / 32; ++w)
            for (int i = 0; i < NB; ++i) {
                if (GI > 0)  // group reads: positions b + rho * R / R_g, b = tb + i * T
                    for (int rho = 0; rho < G.R; ++rho)
                        access<Cfg>("group read", w, [&](int t, int& pt, int& pc) {
                            pt = t / UPC;
                            pc = i * T + rho * (R / G.R);
                        }, unit, total);
                for (int s = 0; s < G.R; ++s) {
                    if (!last) {  // exchange writes: Jl * R_g * ELL + kl + mu * ELL
                        access<Cfg>("exchange write", w, [&](int t, int& pt, int& pc) {
                            const int tb = t / UPC, it = i * T;
                            pt = (tb / ELL) * G.R * ELL + tb % ELL;
                            pc = (it / ELL) * G.R * ELL + it % ELL + group_mu(G, s) * ELL;
                        }, unit, total);
                    } else if (L_IN == 1 && !Cfg::kStoreTMA) {  // first pass: stage the unit rows
                        access<Cfg>("first-pass staging write", w, [&](int t, int& pt, int& pc) {
                            pt = t / UPC;
                            pc = i * T + group_mu(G, s) * ELL;
                        }, unit, total);
                    }
                }
            }
        if (last && L_IN == 1 && !Cfg::kStoreTMA)  // column-wise copy-out
            for (int k = 0; k < UPC * R / Cfg::THREADS; ++k)
                for (int w = 0; w < Cfg::THREADS / 32; ++w)
                    access<Cfg>("copy-out read", w, [&](int t, int& pt, int& pc) {
                        pt = t;
                        pc = (k * Cfg::THREADS) % R;
                    }, [&](int) { return (k * Cfg::THREADS) / R; }, total);
    }
    *bad_out = bad;
    return total;
}

template <typename F, int P, int PI, int S>
void check(const char* name) {
    using Cfg = PassCfg<F, P, PI, S>;
    static_assert(Cfg::KROWS > 1, "a short-row pass");
    int bad = 0;
    const int total = replay<Cfg, P, S>(&bad);
    std::printf("%-34s R %4d, %2d units per CTA, %d rows per line: %s (%d extra wavefronts)\n", name, Cfg::R,
                Cfg::UPC, Cfg::KROWS, (bad || total) ? "FAIL" : "ok", total);
    if (bad || total) ++g_fail;
}

// The padded [position][unit] layout of the 128-byte-row passes, applied to a
// short-row pass: the replay must find its conflicts (a check of the check).
struct Padded18 : PassCfg<float, 18, 0, 0> {
    static constexpr int KROWS = 1;
};

}  // namespace

// Segment tiles of the macro path at micro order M: TPC columns of N points,
// point k of column q at keep_idx(k, q). Writes: the last stage group writes
// consecutive points of one column per thread group; reads: the transposed
// store reads consecutive elements k * TPC + q.
template <typename F, int M>
void check_keep(const char* name) {
    using SC = SegCfg<F, M>;
    using Wk = TileWorker<F, M, kC2CFwd, kAoS, kAoS, SC::BLOCK, false, false, false, true, SC::E>;
    using C = Cx<F>;
    constexpr int N = 1 << M, TPC = Wk::TPC, T = Wk::T, BLOCK = SC::BLOCK;
    constexpr int SL = 128 / (int)sizeof(C), lanes = SL;  // bank groups per line, lanes per phase
    int bad = 0, extra = 0;
    std::set<int> seen;
    for (int k = 0; k < N; ++k)
        for (int q = 0; q < TPC; ++q) {
            const int i = (int)Wk::keep_idx(k, q);
            if (i < 0 || i >= TPC * N || !seen.insert(i).second) ++bad;
        }
    auto phase_extra = [&](const std::vector<int>& idx) {
        for (size_t ph = 0; ph < idx.size(); ph += lanes) {
            std::map<int, std::set<int>> bank;
            for (size_t l = ph; l < ph + lanes && l < idx.size(); ++l) bank[idx[l] % SL].insert(idx[l]);
            int worst = 1;
            for (auto& kv : bank) worst = (int)kv.second.size() > worst ? (int)kv.second.size() : worst;
            extra += worst - 1;
        }
    };
    for (int w = 0; w < BLOCK / 32; ++w) {
        for (int off = 0; off < N; off += T) {  // writes: thread t holds point (t % T) + off of column t / T
            std::vector<int> idx;
            for (int lane = 0; lane < 32; ++lane) {
                const int t = 32 * w + lane;
                idx.push_back((int)Wk::keep_idx(t % T + off, t / T));
            }
            phase_extra(idx);
        }
        for (int e0 = 0; e0 < TPC * N; e0 += BLOCK) {  // reads: element e = k * TPC + q
            std::vector<int> idx;
            for (int lane = 0; lane < 32; ++lane) {
                const int e = e0 + 32 * w + lane;
                idx.push_back((int)Wk::keep_idx(e / TPC, e % TPC));
            }
            phase_extra(idx);
        }
    }
    std::printf("%-34s %2d columns of %5d points: %s (%d extra wavefronts)\n", name, TPC, N,
                (bad || extra) ? "FAIL" : "ok", extra);
    if (bad || extra) ++g_fail;
}

int main() {
    check<float, 17, 0, 0>("CFFT<float> order 17 pass 0");
    check<float, 18, 0, 0>("CFFT<float> order 18 pass 0");
    check<float, 19, 0, 1>("CFFT<float> order 19 pass 0 (two)");
    check<float, 19, 1, 1>("CFFT<float> order 19 pass 1 (two)");
    check<float, 20, 0, 1>("CFFT<float> order 20 pass 0 (two)");
    check<float, 20, 1, 1>("CFFT<float> order 20 pass 1 (two)");
    check<float, 25, 0, 0>("CFFT<float> order 25 pass 0");
    check<float, 26, 0, 0>("CFFT<float> order 26 pass 0");
    check<double, 18, 0, 0>("CFFT<double> order 18 pass 0");
    check<double, 19, 1, 1>("CFFT<double> order 19 pass 1 (two)");
    check<double, 20, 0, 1>("CFFT<double> order 20 pass 0 (two)");
    check<double, 20, 1, 1>("CFFT<double> order 20 pass 1 (two)");
    check<double, 26, 0, 0>("CFFT<double> order 26 pass 0");
    check_keep<float, 8>("segment tiles, float, micro 8");
    check_keep<float, 9>("segment tiles, float, micro 9");
    check_keep<float, 10>("segment tiles, float, micro 10");
    check_keep<float, 11>("segment tiles, float, micro 11");
    check_keep<float, 12>("segment tiles, float, micro 12");
    check_keep<double, 8>("segment tiles, double, micro 8");
    check_keep<double, 9>("segment tiles, double, micro 9");
    check_keep<double, 10>("segment tiles, double, micro 10");
    check_keep<double, 11>("segment tiles, double, micro 11");
    check_keep<double, 12>("segment tiles, double, micro 12");
    int bad = 0;
    g_quiet = true;
    const int padded = replay<Padded18, 18, 0>(&bad);
    std::printf("control: padded rows on CFFT<float> order 18 pass 0: %d extra wavefronts (%s)\n", padded,
                padded > 0 ? "detected" : "NOT DETECTED");
    if (padded == 0) ++g_fail;
    return g_fail ? 1 : 0;
}
