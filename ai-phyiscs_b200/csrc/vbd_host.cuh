// Host side of the cloth VBD solver (the reference's ClothVBDSolver,
// src/bindings.cpp:1868-1957, solver/vbd_solver.h:134-176): colouring,
// per-vertex adjacency, and the step, which runs as one CUDA graph (predictor,
// iterations x colours sweep kernels, velocity update) rebuilt only when the
// step's arguments change.  Included by cloth_sim.cu (shares its error
// handling and device buffers).
#pragma once

#include <numeric>

#include "vbd_kernels.cuh"

namespace chysx_b200 {

class VbdSolver {
public:
    ~VbdSolver() { drop_graph(); }

    // Greedy colouring of the conflict graph (triangle edges and every pair
    // of a bending edge's vertices, vbd_solver.cu:724-811): vertices by
    // decreasing degree, ties by index, each takes the smallest colour its
    // coloured neighbours do not use.
    void build_cloth_coloring(const int32_t* tris, int n_tris, const int32_t* edges, int n_edges, int n) {
        if (n < 0 || n_tris < 0 || n_edges < 0) throw std::invalid_argument("build_cloth_coloring: negative count");
        std::vector<std::vector<int>> adj(n);
        auto link = [&](int u, int w) {
            if (u < 0 || w < 0) return;
            if (u >= n || w >= n) throw std::out_of_range("build_cloth_coloring: vertex index out of range");
            if (u == w) return;
            adj[u].push_back(w);
            adj[w].push_back(u);
        };
        for (int t = 0; t < n_tris; ++t)
            for (int a = 0; a < 3; ++a)
                for (int b = a + 1; b < 3; ++b) link(tris[3 * t + a], tris[3 * t + b]);
        for (int e = 0; e < n_edges; ++e)
            for (int a = 0; a < 4; ++a)
                for (int b = a + 1; b < 4; ++b) link(edges[4 * e + a], edges[4 * e + b]);
        for (auto& l : adj) {
            std::sort(l.begin(), l.end());
            l.erase(std::unique(l.begin(), l.end()), l.end());
        }
        std::vector<int> order(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return adj[a].size() > adj[b].size(); });
        std::vector<int> colors(n, -1), mark;
        for (int v : order) {
            mark.assign(adj[v].size() + 2, 0);
            for (int w : adj[v])
                if (colors[w] >= 0 && colors[w] < (int)mark.size()) mark[colors[w]] = 1;
            int c = 0;
            while (mark[c]) ++c;
            colors[v] = c;
        }
        set_coloring(colors.data(), n);
    }

    // An external colouring (vbd_solver.cu:490-520).
    void set_coloring(const int32_t* colors, int n) {
        if (n < 0) throw std::invalid_argument("set_coloring: negative count");
        if (n > 0 && !colors) throw std::invalid_argument("set_coloring: null colours");
        int nc = 0;
        for (int i = 0; i < n; ++i) {
            if (colors[i] < 0) throw std::invalid_argument("set_coloring: negative colour");
            nc = std::max(nc, colors[i] + 1);
        }
        colors_.assign(colors, colors + n);
        group_off_.assign(nc + 1, 0);
        for (int i = 0; i < n; ++i) ++group_off_[colors[i] + 1];
        for (int c = 0; c < nc; ++c) group_off_[c + 1] += group_off_[c];
        ids_.assign(n, 0);
        std::vector<int> fill(group_off_.begin(), group_off_.end() - 1);
        for (int i = 0; i < n; ++i) ids_[fill[colors[i]]++] = i;  // by vertex index within a colour
        n_ = n;
        dirty_ = true;  // uploaded by the next step
        drop_graph();
    }

    // Per-vertex (element, local vertex) pairs, in element order
    // (vbd_solver.cu:813-911).
    void build_tri_adjacency(const int32_t* tris, int n_tris, int n) {
        build_adjacency(tris, n_tris, 3, n, tri_off_, tri_adj_, "build_tri_adjacency");
    }
    void build_edge_adjacency(const int32_t* edges, int n_edges, int n) {
        build_adjacency(edges, n_edges, 4, n, edge_off_, edge_adj_, "build_edge_adjacency");
    }

    int num_colors() const { return group_off_.empty() ? 0 : (int)group_off_.size() - 1; }
    void colors(int32_t* out, int n) const {
        if (n != (int)colors_.size()) throw std::invalid_argument("colors: wrong particle count");
        std::copy(colors_.begin(), colors_.end(), out);
    }

    // One VBD step (vbd_solver.cu:897-979).
    void step_cloth(uintptr_t pos, uintptr_t vel, uintptr_t inv_mass, int n, uintptr_t tris, uintptr_t poses,
                    uintptr_t areas, uintptr_t mats, int n_tris, uintptr_t edges, uintptr_t rest_angle,
                    uintptr_t rest_length, uintptr_t bend, int n_edges, float gx, float gy, float gz, float dt,
                    int iterations, uintptr_t stream) {
        if (n <= 0) return;
        if (!pos || !vel || !inv_mass) throw std::invalid_argument("step_cloth: pos, vel and inv_mass are required");
        if (!(dt > 0.0f)) throw std::invalid_argument("step_cloth: dt must be positive");
        if (iterations < 0) throw std::invalid_argument("step_cloth: negative iteration count");
        if (n_ != n) throw std::invalid_argument("step_cloth: the colouring covers a different particle count");
        if (n_tris > 0 && (!tris || !poses || !areas || !mats))
            throw std::invalid_argument("step_cloth: triangle arrays are required with n_tris > 0");
        if (n_edges > 0 && (!edges || !rest_angle || !rest_length || !bend))
            throw std::invalid_argument("step_cloth: edge arrays are required with n_edges > 0");
        if (n_tris > 0 && tri_n_ != n) throw std::invalid_argument("step_cloth: build_tri_adjacency first");
        if (n_edges > 0 && edge_n_ != n) throw std::invalid_argument("step_cloth: build_edge_adjacency first");
        if (dirty_) {
            d_ids_.upload(ids_.empty() ? std::vector<int>{0} : ids_);
            if (tri_n_ >= 0) {
                d_tri_off_.upload(tri_off_);
                d_tri_adj_.upload(tri_adj_);
            }
            if (edge_n_ >= 0) {
                d_edge_off_.upload(edge_off_);
                d_edge_adj_.upload(edge_adj_);
            }
            dirty_ = false;
        }
        if (d_q_prev_.size() != 3 * (size_t)n) {
            d_q_prev_.resize(3 * (size_t)n);
            d_inertia_.resize(3 * (size_t)n);
            d_disp_.resize(3 * (size_t)n);
            d_mass_.resize((size_t)n);
            drop_graph();
        }
        vbd::ClothArgs a;
        std::memset(&a, 0, sizeof(a));  // compared bytewise with the graph's
        a.pos = reinterpret_cast<float*>(pos);
        a.vel = reinterpret_cast<float*>(vel);
        a.inv_mass = reinterpret_cast<const float*>(inv_mass);
        a.q_prev = d_q_prev_.get();
        a.inertia = d_inertia_.get();
        a.disp = d_disp_.get();
        a.mass = d_mass_.get();
        a.tris = n_tris > 0 ? reinterpret_cast<const int*>(tris) : nullptr;
        a.poses = n_tris > 0 ? reinterpret_cast<const float*>(poses) : nullptr;
        a.areas = n_tris > 0 ? reinterpret_cast<const float*>(areas) : nullptr;
        a.mats = n_tris > 0 ? reinterpret_cast<const float*>(mats) : nullptr;
        a.tri_off = d_tri_off_.get();
        a.tri_adj = d_tri_adj_.get();
        a.edges = n_edges > 0 ? reinterpret_cast<const int*>(edges) : nullptr;
        a.rest_angle = n_edges > 0 ? reinterpret_cast<const float*>(rest_angle) : nullptr;
        a.rest_length = n_edges > 0 ? reinterpret_cast<const float*>(rest_length) : nullptr;
        a.bend = n_edges > 0 ? reinterpret_cast<const float*>(bend) : nullptr;
        a.edge_off = d_edge_off_.get();
        a.edge_adj = d_edge_adj_.get();
        a.n = n;
        a.gx = gx;
        a.gy = gy;
        a.gz = gz;
        a.dt = dt;
        if (!exec_ || !same_bytes(a, graph_args_) || iterations != graph_iters_) build_graph(a, iterations);
        ck(cudaGraphLaunch(exec_, reinterpret_cast<cudaStream_t>(stream)), "cudaGraphLaunch(vbd step)");
    }

private:
    void build_adjacency(const int32_t* el, int count, int arity, int n, std::vector<int>& off, std::vector<int>& adj,
                         const char* what) {
        if (n < 0 || count < 0) throw std::invalid_argument(std::string(what) + ": negative count");
        if (count > 0 && !el) throw std::invalid_argument(std::string(what) + ": null element array");
        off.assign(n + 1, 0);
        for (int e = 0; e < count; ++e)
            for (int k = 0; k < arity; ++k) {
                const int v = el[arity * e + k];
                if (v < 0) continue;
                if (v >= n) throw std::out_of_range(std::string(what) + ": vertex index out of range");
                off[v + 1] += 2;
            }
        for (int v = 0; v < n; ++v) off[v + 1] += off[v];
        adj.assign(off[n], 0);
        std::vector<int> fill(off.begin(), off.end() - 1);
        for (int e = 0; e < count; ++e)
            for (int k = 0; k < arity; ++k) {
                const int v = el[arity * e + k];
                if (v < 0) continue;
                adj[fill[v]] = e;
                adj[fill[v] + 1] = k;
                fill[v] += 2;
            }
        if (adj.empty()) adj.push_back(0);
        (arity == 3 ? tri_n_ : edge_n_) = n;
        dirty_ = true;
        drop_graph();
    }

    // lanes per vertex: as many (up to 8) as keep the colour's threads within
    // four times what the GPU holds at two 256-thread CTAs per SM
    static int lanes_for(int count) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const long cap = 4L * sms * 512;
        for (int l : {8, 4, 2})
            if ((long)count * l <= cap) return l;
        return 1;
    }

    void drop_graph() {
        if (exec_) cudaGraphExecDestroy(exec_);
        exec_ = nullptr;
    }

    // predictor, iterations x colours sweeps, velocity: all in one graph
    void build_graph(const vbd::ClothArgs& a, int iterations) {
        drop_graph();
        cudaGraph_t g;
        ck(cudaGraphCreate(&g, 0), "cudaGraphCreate(vbd)");
        vbd::ClothArgs args = a;
        cudaGraphNode_t last = nullptr;
        auto add = [&](void* fn, int threads, void** params) {
            cudaKernelNodeParams p{};
            p.func = fn;
            p.gridDim = dim3(std::max(1, grid_for(threads, kVecBlock)));
            p.blockDim = dim3(kVecBlock);
            p.kernelParams = params;
            cudaGraphNode_t node;
            ck(cudaGraphAddKernelNode(&node, g, last ? &last : nullptr, last ? 1 : 0, &p), "add vbd node");
            last = node;
        };
        {
            void* prm[] = {&args};
            add(reinterpret_cast<void*>(&vbd::vbd_forward_kernel), a.n, prm);
        }
        const int nc = num_colors();
        std::vector<const int*> ids(nc);
        std::vector<int> counts(nc);
        for (int it = 0; it < iterations; ++it)
            for (int c = 0; c < nc; ++c) {
                counts[c] = group_off_[c + 1] - group_off_[c];
                if (counts[c] == 0) continue;
                ids[c] = d_ids_.get() + group_off_[c];
                void* prm[] = {&args, &ids[c], &counts[c]};
                const int lanes = lanes_for(counts[c]);
                void* fn = lanes == 8   ? reinterpret_cast<void*>(&vbd::vbd_color_kernel<8>)
                           : lanes == 4 ? reinterpret_cast<void*>(&vbd::vbd_color_kernel<4>)
                           : lanes == 2 ? reinterpret_cast<void*>(&vbd::vbd_color_kernel<2>)
                                        : reinterpret_cast<void*>(&vbd::vbd_color_kernel<1>);
                add(fn, counts[c] * lanes, prm);
            }
        {
            void* prm[] = {&args};
            add(reinterpret_cast<void*>(&vbd::vbd_velocity_kernel), a.n, prm);
        }
        const cudaError_t e = cudaGraphInstantiate(&exec_, g, 0);
        cudaGraphDestroy(g);
        ck(e, "cudaGraphInstantiate(vbd)");
        graph_args_ = a;
        graph_iters_ = iterations;
    }

    int n_ = 0, tri_n_ = -1, edge_n_ = -1;
    std::vector<int> colors_, group_off_;
    std::vector<int> ids_, tri_off_, tri_adj_, edge_off_, edge_adj_;  // host copies, uploaded by step
    bool dirty_ = false;
    DevBuf<int> d_ids_, d_tri_off_, d_tri_adj_, d_edge_off_, d_edge_adj_;
    DevBuf<float> d_q_prev_, d_inertia_, d_disp_, d_mass_;
    cudaGraphExec_t exec_ = nullptr;
    vbd::ClothArgs graph_args_{};
    int graph_iters_ = -1;
};

}  // namespace chysx_b200
