// dv_colour.cu -- host C++: exact stencil pattern of the Jacobian and its greedy distance-2 column
// colouring, identical element for element to the reference (numerics/sparsity.py:29-107):
//   pattern  gas + energy rows of cell (i,j,k) <- all 6 unknowns of (i,j,k), (i,j,k+-1), (i,j,k+-2),
//            (i+-1,j,k), (i,j+-1 mod Nth,k) [+ the wall node of an outer cell]; loading rows <- own
//            cell; wall rows <- wall (j,k), (j,k+-1), (j+-1,k) and the outer cell (Nr-1,j,k);
//   colour   columns visited by decreasing degree in G = P^T P (stable for equal degrees), each given
//            the smallest colour absent from its G-neighbours.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>
#include "dv_internal.h"

namespace {

struct Pattern {
    int64_t n;
    std::vector<int64_t> rptr, rcol;   // CSR
    std::vector<int64_t> cptr, crow;   // CSC
};

void build(int Nr, int Nth, int Nz, bool wall, Pattern& P) {
    const int64_t nc = (int64_t)Nr * Nth * Nz;
    const int64_t nw = wall ? (int64_t)Nth * Nz : 0;
    const int64_t n = DV_NV * nc + nw;
    P.n = n;
    auto cell = [&](int i, int j, int k) { return ((int64_t)i * Nth + j) * Nz + k; };
    std::vector<std::vector<int64_t>> rows((size_t)n);
    std::vector<int64_t> st;
    for (int i = 0; i < Nr; ++i)
        for (int j = 0; j < Nth; ++j)
            for (int k = 0; k < Nz; ++k) {
                const int64_t c = cell(i, j, k);
                st.clear();
                st.push_back(c);
                for (int dk = 1; dk <= 2; ++dk) {
                    if (Nz > dk) {
                        if (k - dk >= 0) st.push_back(cell(i, j, k - dk));
                        if (k + dk < Nz) st.push_back(cell(i, j, k + dk));
                    }
                }
                if (Nr > 1) {
                    if (i > 0) st.push_back(cell(i - 1, j, k));
                    if (i < Nr - 1) st.push_back(cell(i + 1, j, k));
                }
                if (Nth > 1) {
                    st.push_back(cell(i, (j + 1) % Nth, k));
                    st.push_back(cell(i, (j + Nth - 1) % Nth, k));
                }
                const int flux_rows[4] = {0, 1, 2, DV_NV - 1};
                for (int fr : flux_rows) {
                    auto& row = rows[(size_t)(fr * nc + c)];
                    for (int64_t sc : st)
                        for (int v = 0; v < DV_NV; ++v) row.push_back(v * nc + sc);
                    if (wall && i == Nr - 1) row.push_back(DV_NV * nc + (int64_t)j * Nz + k);
                }
                for (int qr = DV_NG; qr < DV_NG + DV_NA; ++qr) {
                    auto& row = rows[(size_t)(qr * nc + c)];
                    for (int v = 0; v < DV_NV; ++v) row.push_back(v * nc + c);
                }
            }
    if (wall) {
        for (int j = 0; j < Nth; ++j)
            for (int k = 0; k < Nz; ++k) {
                const int64_t w = (int64_t)j * Nz + k;
                auto& row = rows[(size_t)(DV_NV * nc + w)];
                row.push_back(DV_NV * nc + w);
                if (Nz > 1) {
                    if (k > 0) row.push_back(DV_NV * nc + w - 1);
                    if (k < Nz - 1) row.push_back(DV_NV * nc + w + 1);
                }
                if (Nth > 1) {
                    row.push_back(DV_NV * nc + (int64_t)((j + 1) % Nth) * Nz + k);
                    row.push_back(DV_NV * nc + (int64_t)((j + Nth - 1) % Nth) * Nz + k);
                }
                const int64_t oc = cell(Nr - 1, j, k);
                for (int v = 0; v < DV_NV; ++v) row.push_back(v * nc + oc);
            }
    }
    P.rptr.assign((size_t)n + 1, 0);
    for (int64_t r = 0; r < n; ++r) {
        auto& row = rows[(size_t)r];
        std::sort(row.begin(), row.end());
        row.erase(std::unique(row.begin(), row.end()), row.end());
        P.rptr[(size_t)r + 1] = P.rptr[(size_t)r] + (int64_t)row.size();
    }
    P.rcol.resize((size_t)P.rptr[(size_t)n]);
    for (int64_t r = 0; r < n; ++r) std::copy(rows[(size_t)r].begin(), rows[(size_t)r].end(), P.rcol.begin() + P.rptr[(size_t)r]);
    P.cptr.assign((size_t)n + 1, 0);
    for (int64_t q : P.rcol) P.cptr[(size_t)q + 1] += 1;
    for (int64_t c = 0; c < n; ++c) P.cptr[(size_t)c + 1] += P.cptr[(size_t)c];
    P.crow.resize(P.rcol.size());
    std::vector<int64_t> pos(P.cptr.begin(), P.cptr.end() - 1);
    for (int64_t r = 0; r < n; ++r)
        for (int64_t e = P.rptr[(size_t)r]; e < P.rptr[(size_t)r + 1]; ++e) P.crow[(size_t)pos[(size_t)P.rcol[(size_t)e]]++] = r;
}

}  // namespace

namespace {
// The colouring depends only on (Nr, Nth, Nz, wall) and takes ~50 ms at 8x8x32; every model of a
// cycle step asks for it (model creation for the colour count, the Jacobian for the colours), so
// each shape is coloured once per process and copied afterwards.
struct ColourKey {
    int32_t Nr, Nth, Nz, wall;
    bool operator<(const ColourKey& o) const {
        return std::tie(Nr, Nth, Nz, wall) < std::tie(o.Nr, o.Nth, o.Nz, o.wall);
    }
};
struct ColourEntry {
    std::vector<int64_t> colour;
    int32_t ncolours;
};
std::mutex g_colour_mu;
std::map<ColourKey, ColourEntry> g_colour_cache;

int colour_columns_uncached(int32_t Nr, int32_t Nth, int32_t Nz, int32_t wall, int64_t* colour, int32_t* ncolours);
}  // namespace

extern "C" int dv_colour_columns(int32_t Nr, int32_t Nth, int32_t Nz, int32_t wall, int64_t* colour, int32_t* ncolours) {
    if (Nr < 1 || Nth < 1 || Nz < 1 || !colour) {
        dv::set_error("dv_colour_columns: bad arguments");
        return DV_ERR_ARG;
    }
    const ColourKey key{Nr, Nth, Nz, wall != 0 ? 1 : 0};
    std::lock_guard<std::mutex> lock(g_colour_mu);
    auto it = g_colour_cache.find(key);
    if (it == g_colour_cache.end()) {
        const int64_t n = (int64_t)6 * Nr * Nth * Nz + (wall ? (int64_t)Nth * Nz : 0);
        ColourEntry e{std::vector<int64_t>((size_t)n), 0};
        const int rc = colour_columns_uncached(Nr, Nth, Nz, key.wall, e.colour.data(), &e.ncolours);
        if (rc != DV_OK) return rc;
        it = g_colour_cache.emplace(key, std::move(e)).first;
    }
    std::memcpy(colour, it->second.colour.data(), it->second.colour.size() * sizeof(int64_t));
    if (ncolours) *ncolours = it->second.ncolours;
    return DV_OK;
}

namespace {
int colour_columns_uncached(int32_t Nr, int32_t Nth, int32_t Nz, int32_t wall, int64_t* colour, int32_t* ncolours) {
    Pattern P;
    build(Nr, Nth, Nz, wall != 0, P);
    const int64_t n = P.n;
    std::vector<int64_t> stamp((size_t)n, -1), deg((size_t)n, 0);
    for (int64_t j = 0; j < n; ++j) {       // degree of column j in G = P^T P (self included)
        int64_t d = 0;
        for (int64_t e = P.cptr[(size_t)j]; e < P.cptr[(size_t)j + 1]; ++e) {
            const int64_t r = P.crow[(size_t)e];
            for (int64_t f = P.rptr[(size_t)r]; f < P.rptr[(size_t)r + 1]; ++f) {
                const int64_t q = P.rcol[(size_t)f];
                if (stamp[(size_t)q] != j) {
                    stamp[(size_t)q] = j;
                    ++d;
                }
            }
        }
        deg[(size_t)j] = d;
    }
    std::vector<int64_t> order((size_t)n);
    for (int64_t j = 0; j < n; ++j) order[(size_t)j] = j;
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return deg[(size_t)a] > deg[(size_t)b]; });
    for (int64_t j = 0; j < n; ++j) colour[j] = -1;
    std::vector<int64_t> used_stamp(1024, -1);
    int64_t maxc = -1;
    std::fill(stamp.begin(), stamp.end(), -1);
    for (int64_t idx = 0; idx < n; ++idx) {
        const int64_t j = order[(size_t)idx];
        for (int64_t e = P.cptr[(size_t)j]; e < P.cptr[(size_t)j + 1]; ++e) {
            const int64_t r = P.crow[(size_t)e];
            for (int64_t f = P.rptr[(size_t)r]; f < P.rptr[(size_t)r + 1]; ++f) {
                const int64_t q = P.rcol[(size_t)f];
                const int64_t cq = colour[q];
                if (cq >= 0) {
                    if ((size_t)cq >= used_stamp.size()) used_stamp.resize((size_t)cq * 2 + 1, -1);
                    used_stamp[(size_t)cq] = idx;
                }
            }
        }
        int64_t c = 0;
        while ((size_t)c < used_stamp.size() && used_stamp[(size_t)c] == idx) ++c;
        colour[j] = c;
        if (c > maxc) maxc = c;
    }
    if (ncolours) *ncolours = (int32_t)(maxc + 1);
    return DV_OK;
}
}  // namespace
