// natural_insert.cpp -- a host program that uses the C ABI the way the
// reference's PETSc runtime would, without PETSc: it assembles the Natural
// Jacobian of a grid through nz_jacobian_columns and inserts every cell's
// column into a block-CSR matrix exactly as insertPreparedCellJacobianColumn_
// does (MatSetValuesBlocked(J, 1 + nnbr, rows, 1, &col, vals, ADD_VALUES) on a
// zeroed matrix; models/include/natural/petsc/detail/
// natural_petsc_runtime_jacobian.inc:279-299), then inserts the row-ordered
// output of nz_jacobian block by block (INSERT_VALUES) into a second matrix,
// and compares both with the reference's captured matrix.
//
// Input: a directory written by tests/test_insert_gpu.py (raw little-endian
// arrays).  Exit code 0 when both matrices agree with the reference within the
// tolerance; prints one summary line.
#include "nonenone_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace
{
template <class T>
std::vector<T> readArray(const std::string &dir, const char *name)
{
    const std::string path = dir + "/" + name;
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f)
    {
        std::fprintf(stderr, "cannot open %s\n", path.c_str());
        std::exit(2);
    }
    std::fseek(f, 0, SEEK_END);
    const long bytes = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<T> v(size_t(bytes) / sizeof(T));
    if (std::fread(v.data(), sizeof(T), v.size(), f) != v.size())
        std::exit(2);
    std::fclose(f);
    return v;
}

// A block-CSR matrix with a fixed pattern: the part of PETSc's BAIJ matrix the
// insertion exercises (MAT_NEW_NONZERO_LOCATION_ERR: a block outside the
// pattern is an error).
struct Bcsr
{
    int B;
    std::vector<int64_t> rowPtr, colIdx;
    std::vector<double> values;

    int64_t find(int64_t row, int64_t col) const
    {
        const auto first = colIdx.begin() + rowPtr[row], last = colIdx.begin() + rowPtr[row + 1];
        const auto it = std::lower_bound(first, last, col);
        return (it != last && *it == col) ? int64_t(it - colIdx.begin()) : -1;
    }
    // MatSetValuesBlocked(m rows, n cols), values row-oriented: the (m*B) x
    // (n*B) dense array, entry (i*B + r, j*B + k) at ((i*B + r) * n + j) * B + k.
    bool setBlocked(int m, const int64_t *rows, int n, const int64_t *cols, const double *v, bool add)
    {
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < n; ++j)
            {
                const int64_t slot = find(rows[i], cols[j]);
                if (slot < 0)
                    return false;
                double *blk = &values[size_t(slot) * B * B];
                for (int r = 0; r < B; ++r)
                    for (int k = 0; k < B; ++k)
                    {
                        const double x = v[((size_t(i) * B + r) * n + j) * B + k];
                        blk[r * B + k] = add ? blk[r * B + k] + x : x;
                    }
            }
        return true;
    }
};

int check(int rc, const char *what)
{
    if (rc < 0)
    {
        std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, nz_last_error());
        std::exit(3);
    }
    return rc;
}

// Largest entry error against the reference, relative to the entry, with the
// floor of 1e-6 x the largest entry of the same equation row of the block row
// (entries that are rounding noise next to their row are compared absolutely).
double compare(const Bcsr &m, const std::vector<double> &ref, int64_t ncell, int B, int64_t *floored)
{
    double worst = 0.0;
    *floored = 0;
    for (int64_t row = 0; row < ncell; ++row)
        for (int r = 0; r < B; ++r)
        {
            double scale = 0.0;
            for (int64_t s = m.rowPtr[row]; s < m.rowPtr[row + 1]; ++s)
                for (int k = 0; k < B; ++k)
                    scale = std::max(scale, std::fabs(ref[(size_t(s) * B + r) * B + k]));
            for (int64_t s = m.rowPtr[row]; s < m.rowPtr[row + 1]; ++s)
                for (int k = 0; k < B; ++k)
                {
                    const size_t e = (size_t(s) * B + r) * B + k;
                    const double a = m.values[e], b = ref[e];
                    const double floor = 1.0e-6 * scale;
                    if (b != 0.0 && std::fabs(b) < floor)
                        ++*floored;
                    const double denom = std::max(std::fabs(b), floor);
                    const double err = denom > 0.0 ? std::fabs(a - b) / denom : std::fabs(a - b);
                    worst = std::max(worst, err);
                }
        }
    return worst;
}
} // namespace

int main(int argc, char **argv)
{
    if (argc < 2)
    {
        std::fprintf(stderr, "usage: %s <case directory>\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const auto fluidBytes = readArray<unsigned char>(dir, "fluid.bin");
    const auto meta = readArray<double>(dir, "meta.bin");   // dt, T, fugacity scaling, 7 relperm values
    const auto porosity = readArray<double>(dir, "porosity.bin");
    const auto volume = readArray<double>(dir, "volume.bin");
    const auto offset = readArray<int64_t>(dir, "conn_offset.bin");
    const auto neighbor = readArray<int64_t>(dir, "conn_neighbor.bin");
    const auto trans = readArray<double>(dir, "conn_trans.bin");
    const auto gravity = readArray<double>(dir, "conn_gravity.bin");
    const auto history = readArray<double>(dir, "primary.bin");
    const auto phaseState = readArray<double>(dir, "phase_state.bin");
    const auto current = readArray<double>(dir, "current.bin");
    const auto reference = readArray<double>(dir, "jacobian.bin");
    if (fluidBytes.size() != sizeof(nz_fluid_desc) || meta.size() != 10)
    {
        std::fprintf(stderr, "bad case files\n");
        return 2;
    }
    nz_fluid_desc fluid;
    std::memcpy(&fluid, fluidBytes.data(), sizeof(fluid));
    const int64_t ncell = int64_t(porosity.size());
    const int B = 3 * fluid.nc + 1;

    nz_ctx *ctx = nullptr;
    check(nz_ctx_create(&fluid, nullptr, 0, &ctx), "nz_ctx_create");
    nz_natural_desc desc{};
    desc.ncell = ncell;
    desc.porosity = porosity.data();
    desc.volume = volume.data();
    desc.conn_offset = offset.data();
    desc.conn_neighbor = neighbor.data();
    desc.conn_trans = trans.data();
    desc.conn_gravity = gravity.data();
    desc.time_step = meta[0];
    desc.temperature = meta[1];
    desc.fugacity_scaling = meta[2];
    desc.relperm = {meta[3], meta[4], meta[5], meta[6], meta[7], meta[8], meta[9]};
    nz_natural *nat = nullptr;
    check(nz_natural_create(ctx, &desc, &nat), "nz_natural_create");

    Bcsr a{B, std::vector<int64_t>(size_t(ncell) + 1), {}, {}};
    int64_t nnzb = 0;
    check(nz_natural_pattern(nat, nullptr, nullptr, &nnzb), "nz_natural_pattern");
    a.colIdx.resize(size_t(nnzb));
    check(nz_natural_pattern(nat, a.rowPtr.data(), a.colIdx.data(), &nnzb), "nz_natural_pattern");
    a.values.assign(size_t(nnzb) * B * B, 0.0);   // MatZeroEntries
    Bcsr rowwise = a;
    if (reference.size() != a.values.size())
    {
        std::fprintf(stderr, "reference has %zu entries, pattern %zu\n", reference.size(), a.values.size());
        return 2;
    }

    const size_t stateBytes = history.size() * sizeof(double), psBytes = phaseState.size() * sizeof(double);
    const size_t valueBytes = a.values.size() * sizeof(double);
    double *dHist = nullptr, *dPs = nullptr, *dCur = nullptr, *dVals = nullptr;
    cudaMalloc(&dHist, stateBytes);
    cudaMalloc(&dPs, psBytes);
    cudaMalloc(&dCur, stateBytes);
    cudaMalloc(&dVals, valueBytes);
    cudaMemcpy(dHist, history.data(), stateBytes, cudaMemcpyHostToDevice);
    cudaMemcpy(dPs, phaseState.data(), psBytes, cudaMemcpyHostToDevice);
    cudaMemcpy(dCur, current.data(), stateBytes, cudaMemcpyHostToDevice);
    check(nz_natural_set_history(nat, dHist, dPs, nullptr), "nz_natural_set_history");

    // 1) column order: one batched block write per cell, as the reference does
    check(nz_jacobian_columns(nat, dCur, dPs, dVals, nullptr, nullptr), "nz_jacobian_columns");
    std::vector<double> columns(a.values.size());
    cudaMemcpy(columns.data(), dVals, valueBytes, cudaMemcpyDeviceToHost);
    std::vector<int64_t> rows;
    for (int64_t c = 0; c < ncell; ++c)
    {
        rows.assign(1, c);
        for (int64_t j = offset[c]; j < offset[c + 1]; ++j)
            rows.push_back(neighbor[j]);
        const double *vals = columns.data() + size_t(c + offset[c]) * B * B;
        if (!a.setBlocked(int(rows.size()), rows.data(), 1, &c, vals, true))
        {
            std::fprintf(stderr, "column of cell %lld leaves the pattern\n", (long long)c);
            return 4;
        }
    }
    // 2) pattern order: each block inserted on its own
    check(nz_jacobian(nat, dCur, dPs, dVals, nullptr, nullptr), "nz_jacobian");
    std::vector<double> blocks(a.values.size());
    cudaMemcpy(blocks.data(), dVals, valueBytes, cudaMemcpyDeviceToHost);
    for (int64_t row = 0; row < ncell; ++row)
        for (int64_t s = a.rowPtr[row]; s < a.rowPtr[row + 1]; ++s)
            if (!rowwise.setBlocked(1, &row, 1, &a.colIdx[size_t(s)], blocks.data() + size_t(s) * B * B, false))
                return 4;

    int64_t floored = 0;
    const double errColumns = compare(a, reference, ncell, B, &floored);
    const double errRows = compare(rowwise, reference, ncell, B, &floored);
    std::printf("cells %lld blocks %lld B %d: column insertion max err %.3e, block insertion max err %.3e, "
                "nonzero entries under the row floor %lld of %zu\n",
                (long long)ncell, (long long)nnzb, B, errColumns, errRows, (long long)floored,
                a.values.size());
    cudaFree(dHist);
    cudaFree(dPs);
    cudaFree(dCur);
    cudaFree(dVals);
    nz_natural_destroy(nat);
    nz_ctx_destroy(ctx);
    return (errColumns <= 1.0e-9 && errRows <= 1.0e-9) ? 0 : 1;
}
