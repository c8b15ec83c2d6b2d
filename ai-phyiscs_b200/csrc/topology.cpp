// Host topology builder; see topology.h for the layout.
#include "topology.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>

namespace chysx_b200 {

namespace {

void check_vertex(int v, int n) {
    if (v < 0 || v >= n)
        throw std::out_of_range("vertex index " + std::to_string(v) + " out of range [0, " +
                                std::to_string(n) + ")");
}

// Lays out per-row variable-length lists as sliced ELL: returns the slice
// offsets and fills `out` (pad value `pad`) through `emit(row, k) -> value`.
template <class Count, class Emit, class T>
void slice_layout(int n, int n_slices, Count count, Emit emit, T pad, std::vector<int>& off,
                  std::vector<T>& out) {
    off.assign(n_slices + 1, 0);
    for (int s = 0; s < n_slices; ++s) {
        int w = 0;
        for (int l = 0; l < kSlice; ++l) {
            const int r = s * kSlice + l;
            if (r < n) w = std::max(w, count(r));
        }
        off[s + 1] = off[s] + w * kSlice;
    }
    out.assign(off.back(), pad);
    for (int s = 0; s < n_slices; ++s) {
        const int w = (off[s + 1] - off[s]) / kSlice;
        for (int l = 0; l < kSlice; ++l) {
            const int r = s * kSlice + l;
            if (r >= n) continue;
            const int c = count(r);
            for (int k = 0; k < c && k < w; ++k) out[off[s] + k * kSlice + l] = emit(r, k);
        }
    }
}

}  // namespace

void build_vertex_triangles(int n, const std::vector<int>& tris, std::vector<int>& off,
                            std::vector<int>& list) {
    const int T = (int)(tris.size() / 3);
    off.assign(n + 1, 0);
    for (int t = 0; t < T; ++t)
        for (int a = 0; a < 3; ++a) {
            check_vertex(tris[3 * t + a], n);
            off[tris[3 * t + a] + 1]++;
        }
    for (int i = 0; i < n; ++i) off[i + 1] += off[i];
    list.assign(off[n], 0);
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (int t = 0; t < T; ++t)
        for (int a = 0; a < 3; ++a) list[fill[tris[3 * t + a]]++] = t;
}

namespace {

void bisect(const float* pos, std::vector<int>& ord, int lo, int hi, int block) {
    const int m = hi - lo;
    if (m <= kSlice) return;
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = lo; k < hi; ++k)
        for (int a = 0; a < 3; ++a) {
            mn[a] = std::min(mn[a], pos[3 * (size_t)ord[k] + a]);
            mx[a] = std::max(mx[a], pos[3 * (size_t)ord[k] + a]);
        }
    int ax = 0;
    for (int a = 1; a < 3; ++a)
        if (mx[a] - mn[a] > mx[ax] - mn[ax]) ax = a;
    const int unit = m > 2 * block ? block : kSlice;
    int left = (m / 2 + unit - 1) / unit * unit;
    if (left >= m) left = (m - 1) / kSlice * kSlice;
    if (left <= 0) return;
    auto less = [&](int a, int b) {
        const float pa = pos[3 * (size_t)a + ax], pb = pos[3 * (size_t)b + ax];
        return pa < pb || (pa == pb && a < b);
    };
    std::nth_element(ord.begin() + lo, ord.begin() + lo + left, ord.begin() + hi, less);
    bisect(pos, ord, lo, lo + left, block);
    bisect(pos, ord, lo + left, hi, block);
}

}  // namespace

void spatial_order(const float* pos, int n, const std::vector<int>& inst_offsets, std::vector<int>& order,
                   int block) {
    order.resize(n);
    for (int k = 0; k < n; ++k) order[k] = k;
    if (inst_offsets.empty()) {
        bisect(pos, order, 0, n, block);
        return;
    }
    for (size_t b = 0; b + 1 < inst_offsets.size(); ++b) bisect(pos, order, inst_offsets[b], inst_offsets[b + 1], block);
}

void build_plan(const std::vector<int>& inst_slice, int grid, HostPlan& o) {
    o = HostPlan();
    const int n_inst = (int)inst_slice.size() - 1;
    if (n_inst < 1) throw std::invalid_argument("build_plan: no instances");
    const int n_slices = inst_slice.back();
    for (int b = 0; b < n_inst; ++b)
        if (inst_slice[b + 1] <= inst_slice[b]) throw std::invalid_argument("build_plan: empty instance");
    grid = std::max(1, std::min(grid, n_slices));
    o.grid = grid;
    o.n_inst = n_inst;
    o.inst_slice = inst_slice;
    o.slice_inst.resize(n_slices);
    for (int b = 0; b < n_inst; ++b)
        for (int s = inst_slice[b]; s < inst_slice[b + 1]; ++s) o.slice_inst[s] = b;
    o.cta_slice.resize(grid + 1);
    for (int c = 0; c <= grid; ++c) o.cta_slice[c] = (int)((long long)c * n_slices / grid);
    o.cta_inst_lo.resize(grid);
    o.cta_inst_hi.resize(grid);
    o.inst_cta_lo.assign(n_inst, -1);
    std::vector<int> inst_cta_hi(n_inst, -1);
    for (int c = 0; c < grid; ++c) {
        const int s0 = o.cta_slice[c], s1 = o.cta_slice[c + 1];
        o.max_slices_per_cta = std::max(o.max_slices_per_cta, s1 - s0);
        o.cta_inst_lo[c] = o.slice_inst[s0];
        o.cta_inst_hi[c] = o.slice_inst[s1 - 1];
        o.max_inst_per_cta = std::max(o.max_inst_per_cta, o.cta_inst_hi[c] - o.cta_inst_lo[c] + 1);
        for (int b = o.cta_inst_lo[c]; b <= o.cta_inst_hi[c]; ++b) {
            if (o.inst_cta_lo[b] < 0) o.inst_cta_lo[b] = c;
            inst_cta_hi[b] = c;
        }
    }
    o.inst_slot.assign(n_inst + 1, 0);
    for (int b = 0; b < n_inst; ++b) o.inst_slot[b + 1] = o.inst_slot[b] + (inst_cta_hi[b] - o.inst_cta_lo[b] + 1);
}

void build_dihedrals(const std::vector<int>& tris, std::vector<int>& out) {
    out.clear();
    const int T = (int)(tris.size() / 3);
    std::map<std::pair<int, int>, int> third;  // directed edge -> third vertex
    for (int t = 0; t < T; ++t) {
        const int v[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
        for (int a = 0; a < 3; ++a) third[{v[a], v[(a + 1) % 3]}] = v[(a + 2) % 3];
    }
    for (const auto& kv : third) {
        const int v0 = kv.first.first, v1 = kv.first.second;
        if (v0 >= v1) continue;  // each undirected edge once
        auto rev = third.find({v1, v0});
        if (rev == third.end()) continue;  // boundary edge
        out.insert(out.end(), {v0, v1, kv.second, rev->second});
    }
}

void build_topology(int n_ext, const std::vector<int>& tris_ext, bool use_tris,
                    const std::vector<int>& edges_ext, bool use_springs,
                    const std::vector<int>& pins_ext, const std::vector<int>& inst_offsets,
                    HostTopology& o, const std::vector<int>& dih_ext, bool use_bending,
                    const std::vector<int>& order) {
    if (n_ext < 0) throw std::invalid_argument("negative particle count");
    o = HostTopology();
    o.n_ext = n_ext;
    const int T = use_tris ? (int)(tris_ext.size() / 3) : 0;
    const int E = use_springs ? (int)(edges_ext.size() / 2) : 0;
    const int D = use_bending ? (int)(dih_ext.size() / 4) : 0;
    for (int q = 0; q < 3 * T; ++q) check_vertex(tris_ext[q], n_ext);
    for (int q = 0; q < 2 * E; ++q) check_vertex(edges_ext[q], n_ext);
    for (int q = 0; q < 4 * D; ++q) check_vertex(dih_ext[q], n_ext);
    for (int v : pins_ext) check_vertex(v, n_ext);

    // ---- internal row layout
    int n = n_ext;
    if (!order.empty() && (int)order.size() != n_ext)
        throw std::invalid_argument("row order must list every particle once");
    // a row order without instances is one instance over all particles
    const std::vector<int> whole = {0, n_ext};
    const std::vector<int>& offs = inst_offsets.empty() && !order.empty() ? whole : inst_offsets;
    const int n_inst = offs.empty() ? 1 : (int)offs.size() - 1;
    std::vector<int> inst_of;  // instance of every particle (mapped layouts only)
    if (!offs.empty()) {
        if (n_inst < 1 || offs.front() != 0 || offs.back() != n_ext)
            throw std::invalid_argument("instance offsets must run from 0 to the particle count");
        o.ext_to_row.assign(n_ext, -1);
        inst_of.resize(n_ext);
        o.inst_slice.assign(n_inst + 1, 0);
        int row = 0;
        for (int b = 0; b < n_inst; ++b) {
            const int lo = offs[b], hi = offs[b + 1];
            if (hi <= lo) throw std::invalid_argument("instance offsets must be strictly increasing");
            for (int k = lo; k < hi; ++k) {
                const int e = order.empty() ? k : order[k];
                if (e < lo || e >= hi || o.ext_to_row[e] >= 0)
                    throw std::invalid_argument("row order is not a permutation within every instance");
                o.ext_to_row[e] = row + (k - lo);
                inst_of[e] = b;
            }
            row += ((hi - lo) + kSlice - 1) / kSlice * kSlice;
            o.inst_slice[b + 1] = row / kSlice;
        }
        n = row;
        o.row_to_ext.assign(n, -1);
        for (int e = 0; e < n_ext; ++e) o.row_to_ext[o.ext_to_row[e]] = e;
        for (int t = 0; t < T; ++t) {
            const int b = inst_of[tris_ext[3 * t]];
            if (inst_of[tris_ext[3 * t + 1]] != b || inst_of[tris_ext[3 * t + 2]] != b)
                throw std::invalid_argument("triangle " + std::to_string(t) + " connects two instances");
        }
        for (int d = 0; d < D; ++d) {
            const int b = inst_of[dih_ext[4 * d]];
            for (int a = 1; a < 4; ++a)
                if (inst_of[dih_ext[4 * d + a]] != b)
                    throw std::invalid_argument("dihedral " + std::to_string(d) + " connects two instances");
        }
    }
    auto R = [&](int e) { return o.ext_to_row.empty() ? e : o.ext_to_row[e]; };
    std::vector<int> tris(3 * (size_t)T), edges(2 * (size_t)E), pins(pins_ext.size()), dih(4 * (size_t)D);
    for (int q = 0; q < 4 * D; ++q) dih[q] = R(dih_ext[q]);
    for (int q = 0; q < 3 * T; ++q) tris[q] = R(tris_ext[q]);
    for (int q = 0; q < 2 * E; ++q) edges[q] = R(edges_ext[q]);
    for (size_t q = 0; q < pins.size(); ++q) pins[q] = R(pins_ext[q]);
    o.n = n;
    o.n_slices = (n + kSlice - 1) / kSlice;
    o.n_pad = o.n_slices * kSlice;
    if (inst_offsets.empty()) o.inst_slice = {0, std::max(1, o.n_slices)};

    // ---- adjacency: triangle pairs (src/cloth/cloth_simulator.cu:720-739)
    // plus spring edges, per-row sort + unique (src/sparse/block_csr.cu:111-135)
    std::vector<int> raw_off(n + 1, 0);
    for (int t = 0; t < T; ++t) {
        const int* v = &tris[3 * t];
        for (int a = 0; a < 3; ++a) check_vertex(v[a], n);
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                if (a != b && v[a] != v[b]) raw_off[v[a] + 1]++;
    }
    for (int e = 0; e < E; ++e) {
        const int a = edges[2 * e], b = edges[2 * e + 1];
        check_vertex(a, n);
        check_vertex(b, n);
        if (a != b) { raw_off[a + 1]++; raw_off[b + 1]++; }
    }
    // bending dihedrals: every vertex pair (cloth_simulator.cu:745-757)
    for (int d = 0; d < D; ++d) {
        const int* v = &dih[4 * d];
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b)
                if (a != b && v[a] != v[b]) raw_off[v[a] + 1]++;
    }
    for (int i = 0; i < n; ++i) raw_off[i + 1] += raw_off[i];
    std::vector<int> raw(raw_off[n]);
    {
        std::vector<int> fill(raw_off.begin(), raw_off.end() - 1);
        for (int t = 0; t < T; ++t) {
            const int* v = &tris[3 * t];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    if (a != b && v[a] != v[b]) raw[fill[v[a]]++] = v[b];
        }
        for (int e = 0; e < E; ++e) {
            const int a = edges[2 * e], b = edges[2 * e + 1];
            if (a != b) { raw[fill[a]++] = b; raw[fill[b]++] = a; }
        }
        for (int d = 0; d < D; ++d) {
            const int* v = &dih[4 * d];
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b)
                    if (a != b && v[a] != v[b]) raw[fill[v[a]]++] = v[b];
        }
    }
    o.csr_ptr.assign(n + 1, 0);
    o.csr_col.clear();
    o.csr_col.reserve(raw.size() / 2 + 1);
    for (int i = 0; i < n; ++i) {
        auto b = raw.begin() + raw_off[i], e = raw.begin() + raw_off[i + 1];
        std::sort(b, e);
        auto last = std::unique(b, e);
        const int deg = (int)(last - b);
        if (deg > kMaxRowWidth)
            throw std::runtime_error("particle " + std::to_string(i) + " has " + std::to_string(deg) +
                                     " neighbours; at most " + std::to_string(kMaxRowWidth) +
                                     " are supported");
        o.csr_col.insert(o.csr_col.end(), b, last);
        o.csr_ptr[i + 1] = (int)o.csr_col.size();
    }
    auto deg = [&](int r) { return o.csr_ptr[r + 1] - o.csr_ptr[r]; };
    auto slot_of = [&](int r, int c) -> unsigned {
        if (r == c) return kDiagSlot;
        auto b = o.csr_col.begin() + o.csr_ptr[r], e = o.csr_col.begin() + o.csr_ptr[r + 1];
        auto it = std::lower_bound(b, e, c);
        if (it == e || *it != c) throw std::logic_error("topology: missing (row, col) pair");
        return (unsigned)(it - b);
    };

    // ---- sliced ELL matrix pattern; pads point at the row itself
    slice_layout(n, o.n_slices, deg, [&](int r, int k) { return o.csr_col[o.csr_ptr[r] + k]; }, 0,
                 o.slice_off, o.col);
    for (int s = 0; s < o.n_slices; ++s) {
        const int w = (o.slice_off[s + 1] - o.slice_off[s]) / kSlice;
        o.max_width = std::max(o.max_width, w);
        for (int l = 0; l < kSlice; ++l) {
            const int r = s * kSlice + l;
            const int d = r < n ? deg(r) : 0;
            for (int k = d; k < w; ++k) o.col[o.slice_off[s] + k * kSlice + l] = r;
        }
    }
    o.csr_to_ell.assign(o.csr_col.size(), 0);
    for (int r = 0; r < n; ++r) {
        const int s = r / kSlice, l = r % kSlice;
        for (int k = 0; k < deg(r); ++k) o.csr_to_ell[o.csr_ptr[r] + k] = o.slice_off[s] + k * kSlice + l;
    }

    // ---- triangle incidence (sorted by triangle id per row)
    {
        std::vector<int> cnt_off(n + 1, 0);
        for (int t = 0; t < T; ++t)
            for (int a = 0; a < 3; ++a) cnt_off[tris[3 * t + a] + 1]++;
        for (int i = 0; i < n; ++i) cnt_off[i + 1] += cnt_off[i];
        std::vector<int> ids(cnt_off[n]);
        std::vector<uint32_t> meta(cnt_off[n]);
        std::vector<int> fill(cnt_off.begin(), cnt_off.end() - 1);
        for (int t = 0; t < T; ++t) {
            const int* v = &tris[3 * t];
            for (int a = 0; a < 3; ++a) {
                const int r = v[a];
                const unsigned s1 = slot_of(r, v[(a + 1) % 3]);
                const unsigned s2 = slot_of(r, v[(a + 2) % 3]);
                ids[fill[r]] = t;
                meta[fill[r]] = (unsigned)a | (s1 << 8) | (s2 << 16);
                fill[r]++;
            }
        }
        auto cnt = [&](int r) { return cnt_off[r + 1] - cnt_off[r]; };
        slice_layout(n, o.n_slices, cnt, [&](int r, int k) { return ids[cnt_off[r] + k]; }, -1,
                     o.tinc_off, o.tinc);
        std::vector<int> dummy_off;
        slice_layout(n, o.n_slices, cnt, [&](int r, int k) { return meta[cnt_off[r] + k]; }, 0u,
                     dummy_off, o.tinc_meta);
    }
    // ---- spring incidence
    {
        std::vector<int> cnt_off(n + 1, 0);
        for (int e = 0; e < E; ++e) {
            cnt_off[edges[2 * e] + 1]++;
            cnt_off[edges[2 * e + 1] + 1]++;
        }
        for (int i = 0; i < n; ++i) cnt_off[i + 1] += cnt_off[i];
        std::vector<int> ids(cnt_off[n]);
        std::vector<uint32_t> meta(cnt_off[n]);
        std::vector<int> fill(cnt_off.begin(), cnt_off.end() - 1);
        for (int e = 0; e < E; ++e) {
            const int a = edges[2 * e], b = edges[2 * e + 1];
            ids[fill[a]] = e;
            meta[fill[a]] = 0u | (slot_of(a, b) << 8);
            fill[a]++;
            ids[fill[b]] = e;
            meta[fill[b]] = 1u | (slot_of(b, a) << 8);
            fill[b]++;
        }
        auto cnt = [&](int r) { return cnt_off[r + 1] - cnt_off[r]; };
        slice_layout(n, o.n_slices, cnt, [&](int r, int k) { return ids[cnt_off[r] + k]; }, -1,
                     o.sinc_off, o.sinc);
        std::vector<int> dummy_off;
        slice_layout(n, o.n_slices, cnt, [&](int r, int k) { return meta[cnt_off[r] + k]; }, 0u,
                     dummy_off, o.sinc_meta);
    }
    // ---- dihedral incidence (sorted by dihedral id per row)
    {
        std::vector<int> cnt_off(n + 1, 0);
        for (int d = 0; d < D; ++d)
            for (int a = 0; a < 4; ++a) cnt_off[dih[4 * d + a] + 1]++;
        for (int i = 0; i < n; ++i) cnt_off[i + 1] += cnt_off[i];
        std::vector<int> ids(cnt_off[n]);
        std::vector<uint32_t> meta(cnt_off[n]);
        std::vector<int> fill(cnt_off.begin(), cnt_off.end() - 1);
        for (int d = 0; d < D; ++d) {
            const int* v = &dih[4 * d];
            for (int a = 0; a < 4; ++a) {
                const int r = v[a];
                uint32_t m = (uint32_t)a;
                for (int q = 1; q <= 3; ++q) m |= slot_of(r, v[(a + q) % 4]) << (8 * q);
                ids[fill[r]] = d;
                meta[fill[r]] = m;
                fill[r]++;
            }
        }
        auto cnt = [&](int r) { return cnt_off[r + 1] - cnt_off[r]; };
        slice_layout(n, o.n_slices, cnt, [&](int r, int k) { return ids[cnt_off[r] + k]; }, -1,
                     o.dinc_off, o.dinc);
        std::vector<int> dummy_off;
        slice_layout(n, o.n_slices, cnt, [&](int r, int k) { return meta[cnt_off[r] + k]; }, 0u,
                     dummy_off, o.dinc_meta);
    }
    // ---- pins sorted by row, per-slice ranges
    {
        const int P = (int)pins.size();
        for (int c = 0; c < P; ++c) check_vertex(pins[c], n);
        o.pin_perm.resize(P);
        for (int c = 0; c < P; ++c) o.pin_perm[c] = c;
        std::stable_sort(o.pin_perm.begin(), o.pin_perm.end(),
                         [&](int a, int b) { return pins[a] < pins[b]; });
        o.pin_row.resize(P);
        for (int c = 0; c < P; ++c) o.pin_row[c] = pins[o.pin_perm[c]];
        o.pin_off.assign(o.n_slices + 1, 0);
        for (int c = 0; c < P; ++c) o.pin_off[o.pin_row[c] / kSlice + 1]++;
        for (int s = 0; s < o.n_slices; ++s) o.pin_off[s + 1] += o.pin_off[s];
    }
}

}  // namespace chysx_b200
