// Host build of the device flash headers (they compile as plain C++).
//
//   host_flash DIR MODE
//
// DIR holds fluid.bin (nz_fluid_desc), opts.bin (nz_flash_options), P.bin,
// T.bin, z.bin (nc x n, component-major) and optionally sal.bin, all raw.
// MODE "plain": flash<true> of every point; writes presence.bin (uint8),
// status.bin (uint8) and beta.bin (3 x n) into DIR.
// MODE "memo": every point twice -- once as is, once with its SW allocation
// search precomputed seed by seed into an AllocMemo (the staged kernels'
// lane form) -- and prints the number of points whose answers differ in any
// bit, and how many points read their memo (those whose answer changes when
// every seed of the memo is made inadmissible); likewise the role-permutation
// search stopped where it starts, run ahead into a PermMemo and replayed
// (and how many points reached it).
#include "nonenone_b200.h"
#include "fluid_dev.cuh"
#include "staged.cuh"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

using namespace nz;

template <class T>
static std::vector<T> readBin(const std::string &dir, const char *name)
{
    std::ifstream f(dir + "/" + name, std::ios::binary | std::ios::ate);
    if (!f)
        return {};
    const size_t bytes = size_t(f.tellg());
    f.seekg(0);
    std::vector<T> v(bytes / sizeof(T));
    f.read(reinterpret_cast<char *>(v.data()), std::streamsize(bytes));
    return v;
}

template <class T>
static void writeBin(const std::string &dir, const char *name, const std::vector<T> &v)
{
    std::ofstream f(dir + "/" + name, std::ios::binary);
    f.write(reinterpret_cast<const char *>(v.data()), std::streamsize(v.size() * sizeof(T)));
}

template <int NC>
static bool sameResult(const Result<NC> &a, const Result<NC> &b)
{
    if (a.converged != b.converged || a.presence != b.presence)
        return false;
    for (int p = 0; p < 3; ++p)
    {
        if (a.beta[p] != b.beta[p] || a.sat[p] != b.sat[p] || a.Z[p] != b.Z[p])
            return false;
        for (int i = 0; i < NC; ++i)
            if (a.x[p][i] != b.x[p][i])
                return false;
    }
    return true;
}

template <int NC>
static int run(const std::string &dir, const FluidDev &F, bool memoMode)
{
    const auto P = readBin<double>(dir, "P.bin"), T = readBin<double>(dir, "T.bin");
    const auto z = readBin<double>(dir, "z.bin"), sal = readBin<double>(dir, "sal.bin");
    const size_t n = P.size();
    if (T.size() != n || z.size() != n * NC || (!sal.empty() && sal.size() != n))
    {
        std::fprintf(stderr, "inconsistent inputs\n");
        return 2;
    }
    std::vector<uint8_t> presence(n), status(n);
    std::vector<double> beta(3 * n);
    long differ = 0, replayed = 0, permuted = 0;
    for (size_t i = 0; i < n; ++i)
    {
        double zi[NC];
        for (int c = 0; c < NC; ++c)
            zi[c] = z[c * n + i];
        const double s0 = sal.empty() ? F.salinity : sal[i];
        Solver<NC> s;
        s.setup(&F, s0);
        Result<NC> r;
        s.template flash<true>(P[i], T[i], zi, r);
        const int st = s.err ? s.err : (r.converged ? NZ_FLASH_CONVERGED : NZ_FLASH_FAILED);
        presence[i] = r.converged ? r.presence : 0;
        status[i] = uint8_t(st);
        for (int p = 0; p < 3; ++p)
            beta[p * n + i] = r.converged ? r.beta[p] : 0.0;
        if (!memoMode || F.eosModel != EOS_SW)
            continue;
        // the memo the staged kernels would build: the allocation search's
        // input is the normalised composition
        AllocMemo<NC> memo{};
        double zn[NC];
        for (int c = 0; c < NC; ++c)
            zn[c] = zi[c];
        Solver<NC> prep;
        prep.setup(&F, s0);
        prep.normalize(zn);
        memo.P = P[i];
        memo.T = T[i];
        memo.salinity = s0;
        for (int c = 0; c < NC; ++c)
            memo.z[c] = zn[c];
        memo.valid = 1;
        for (int k = 0; k < kAllocSeedCount; ++k)
        {
            Solver<NC> lane;
            lane.setup(&F, s0);
            lane.allocationSeedOutcome(P[i], T[i], zn, k, memo.seed[k]);
        }
        Solver<NC> m;
        m.setup(&F, s0);
        m.allocMemo = &memo;
        Result<NC> rm;
        m.template flash<true>(P[i], T[i], zi, rm);
        if (m.err != s.err || !sameResult(r, rm))
            ++differ;
        // the role-permutation search the same way: stop where it starts,
        // run every permutation ahead into a PermMemo, then replay it
        Solver<NC> stop;
        stop.setup(&F, s0);
        stop.allocMemo = &memo;
        stop.stopAtPermutations = true;
        Result<NC> rs;
        stop.template flash<true>(P[i], T[i], zi, rs);
        if (stop.reachedPermutations)
        {
            ++permuted;
            PermMemo<NC> pm{};
            pm.P = P[i];
            pm.T = T[i];
            pm.salinity = s0;
            for (int c = 0; c < NC; ++c)
                pm.z[c] = zn[c];
            pm.valid = 1;
            for (int k = 0; k < 6; ++k)
            {
                Solver<NC> w;
                w.setup(&F, s0);
                bool ok = false;
                double g = 0.0;
                w.permutedFlash(P[i], T[i], zn, k, pm.perm[k].r, ok, g);
                pm.perm[k].ok = ok ? 1 : 0;
                pm.perm[k].gibbs = g;
                pm.perm[k].err = w.err;
            }
            Solver<NC> rp;
            rp.setup(&F, s0);
            rp.allocMemo = &memo;
            rp.permMemo = &pm;
            Result<NC> rr;
            rp.template flash<true>(P[i], T[i], zi, rr);
            if (rp.err != s.err || !sameResult(r, rr))
                ++differ;
        }
        // the points whose search read the memo: a memo in which no seed is
        // admissible changes exactly their answers
        AllocMemo<NC> empty = memo;
        for (int k = 0; k < kAllocSeedCount; ++k)
        {
            empty.seed[k].admissible = 0;
            empty.seed[k].err = 0;
        }
        Solver<NC> e;
        e.setup(&F, s0);
        e.allocMemo = &empty;
        Result<NC> re;
        e.template flash<true>(P[i], T[i], zi, re);
        if (e.err != s.err || !sameResult(r, re))
            ++replayed;
    }
    writeBin(dir, "presence.bin", presence);
    writeBin(dir, "status.bin", status);
    writeBin(dir, "beta.bin", beta);
    if (memoMode)
        std::printf("points %zu differ %ld memos %ld permuted %ld\n", n, differ, replayed, permuted);
    else
        std::printf("points %zu\n", n);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 3)
    {
        std::fprintf(stderr, "usage: host_flash DIR plain|memo\n");
        return 2;
    }
    const std::string dir = argv[1];
    const bool memoMode = std::strcmp(argv[2], "memo") == 0;
    const auto fb = readBin<char>(dir, "fluid.bin");
    const auto ob = readBin<char>(dir, "opts.bin");
    if (fb.size() != sizeof(nz_fluid_desc) || ob.size() != sizeof(nz_flash_options))
    {
        std::fprintf(stderr, "fluid.bin / opts.bin have the wrong size\n");
        return 2;
    }
    nz_fluid_desc fd;
    nz_flash_options fo;
    std::memcpy(&fd, fb.data(), sizeof fd);
    std::memcpy(&fo, ob.data(), sizeof fo);
    const FluidDev F = makeFluidDev(fd, fo);
    switch (fd.nc)
    {
    case 3: return run<3>(dir, F, memoMode);
    case 6: return run<6>(dir, F, memoMode);
    default: std::fprintf(stderr, "nc=%d not built here\n", fd.nc); return 2;
    }
}
