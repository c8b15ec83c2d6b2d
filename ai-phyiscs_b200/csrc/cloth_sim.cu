// Host orchestration of the B200-native cloth step and its C ABI
// (include/chysx_cloth.h).
//
// One step() is one CUDA-graph launch.  Default (persistent) path:
//
//   assemble ─ reset ─ pcg_persistent (cooperative, all iterations) ─ finalize
//
// Alternative (loop) path, kept for A/B measurement:
//
//   assemble ─┬─(warm start)─ warm_init ─ warm_fixup ─┐
//             └───────────────(zero guess)────────────┴─ WHILE(cond) { pcg_spmv ; pcg_update } ─ finalize
//
// In the loop path the WHILE node's condition is written on the device by the
// last block of each grid reduction (converged, max_iter, or NaN).  Either way
// the whole step runs with no host round trip and exactly as many iterations
// as the solve needs.
// The graph is built once per topology / solver-mode change; per-step values
// (dt, caller pointers) are patched into the two kernel nodes that read them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/chysx_cloth.h"
#include "../../include/chysx_vbd.h"
#include "cloth_kernels.cuh"
#include "pcg_persistent.cuh"
#include "topology.h"
#include "warm_mlp.cuh"

namespace chysx_b200 {

namespace {

thread_local std::string g_err;

struct CudaFailure : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaFailure(std::string("chysx: ") + what + " failed: " + cudaGetErrorString(e));
}

template <class T>
class DevBuf {
public:
    DevBuf() = default;
    ~DevBuf() { reset(); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    void resize(size_t n) {
        if (n == n_) return;
        reset();
        if (n) ck(cudaMalloc(reinterpret_cast<void**>(&p_), n * sizeof(T)), "cudaMalloc");
        n_ = n;
    }
    void upload(const T* h, size_t n) {
        resize(n);
        if (n) ck(cudaMemcpy(p_, h, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
    }
    void upload(const std::vector<T>& v) { upload(v.data(), v.size()); }
    void zero() {
        if (n_) ck(cudaMemset(p_, 0, n_ * sizeof(T)), "cudaMemset");
    }
    void reset() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    T* get() const { return p_; }
    size_t size() const { return n_; }

private:
    T* p_ = nullptr;
    size_t n_ = 0;
};

constexpr int kVecBlock = 256;
int grid_for(int n, int block) { return (n + block - 1) / block; }

template <class T>
bool same_bytes(const T& a, const T& b) {
    return std::memcmp(&a, &b, sizeof(T)) == 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// Network training entry points (stateless, device pointers)
// ---------------------------------------------------------------------------
constexpr size_t kWsAlign = 256;
size_t align_up(size_t v) { return (v + kWsAlign - 1) / kWsAlign * kWsAlign; }
int train_blocks(int rows) { return std::max(1, std::min(1184, (rows + 16 * kTrainWarps - 1) / (16 * kTrainWarps))); }

// The training kernel's dynamic shared memory is above the 48 KB default, and
// that limit is a per-device function attribute: set it once on every device
// that launches the kernel (the current device), under a lock.
constexpr int kMaxDevices = 64;
std::mutex g_dev_mu;
bool g_train_smem_set[kMaxDevices] = {};

int current_device() {
    int dev = -1;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) throw std::out_of_range("device ordinal beyond 63");
    return dev;
}

void ensure_train_smem() {
    const int dev = current_device();
    std::lock_guard<std::mutex> lock(g_dev_mu);
    if (!g_train_smem_set[dev]) {
        ck(cudaFuncSetAttribute(mlp_train_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem),
           "cudaFuncSetAttribute(mlp_train_tile_kernel)");
        g_train_smem_set[dev] = true;
    }
}

// the weight-gradient kernel's per-chunk partials: a 64 x 64 block and 64 biases per kDwRows rows
size_t dw_partial_bytes(int rows) {
    return (size_t)((std::max(rows, 1) + kDwRows - 1) / kDwRows) * (64 * 64 + 64) * sizeof(float);
}

size_t mlp_workspace_bytes(int rows) {
    const size_t r = (size_t)std::max(rows, 1);
    return align_up(sizeof(MlpPacked)) + 8 * align_up(r * 64 * sizeof(__nv_bfloat16)) +
           align_up((size_t)train_blocks(rows) * kTrainWarps * sizeof(double)) + align_up(dw_partial_bytes(rows));
}

// Forward + backward (when targets != 0) of rows feature vectors; grads in
// the flat parameter layout (normalisation entries zero); optional predicted
// dv output.  Loss = mean squared error of the standardised outputs.
void mlp_gradients(uintptr_t params, uintptr_t features, uintptr_t targets, int rows, uintptr_t grad, double* loss,
                   uintptr_t dv_out, uintptr_t workspace, uint64_t ws_bytes, uintptr_t stream_u) {
    if (rows <= 0) throw std::invalid_argument("mlp: rows must be positive");
    if (!params || !features || !workspace) throw std::invalid_argument("mlp: null device pointer");
    if (ws_bytes < mlp_workspace_bytes(rows)) throw std::invalid_argument("mlp: workspace too small");
    if (targets && !grad) throw std::invalid_argument("mlp: gradients need an output buffer");
    auto stream = reinterpret_cast<cudaStream_t>(stream_u);
    unsigned char* ws = reinterpret_cast<unsigned char*>(workspace);
    MlpPacked* packed = reinterpret_cast<MlpPacked*>(ws);
    size_t off = align_up(sizeof(MlpPacked));
    MlpTrainBufs bufs;
    const size_t mat = align_up((size_t)rows * 64 * sizeof(__nv_bfloat16));
    for (int l = 0; l < 4; ++l) {
        bufs.act[l] = reinterpret_cast<__nv_bfloat16*>(ws + off);
        off += mat;
    }
    for (int l = 0; l < 4; ++l) {
        bufs.dz[l] = reinterpret_cast<__nv_bfloat16*>(ws + off);
        off += mat;
    }
    bufs.sse = reinterpret_cast<double*>(ws + off);
    off += align_up((size_t)train_blocks(rows) * kTrainWarps * sizeof(double));
    const int chunks = (rows + kDwRows - 1) / kDwRows;
    float* part_w = reinterpret_cast<float*>(ws + off);
    float* part_b = part_w + (size_t)chunks * 64 * 64;
    bufs.out = reinterpret_cast<float*>(dv_out);
    mlp_pack_kernel<<<8, 256, 0, stream>>>(reinterpret_cast<const float*>(params), packed);
    ck(cudaGetLastError(), "mlp_pack_kernel launch");
    ensure_train_smem();
    const int blocks = train_blocks(rows);
    // with no targets the kernel still runs the backward on zero residuals;
    // a zero-target buffer is not needed because target rows are only read
    // when targets != 0
    mlp_train_tile_kernel<<<blocks, kTrainWarps * 32, kTrainSmem, stream>>>(
        packed, reinterpret_cast<const float*>(features), reinterpret_cast<const float*>(targets), rows,
        2.0f / (3.0f * (float)rows), bufs);
    ck(cudaGetLastError(), "mlp_train_tile_kernel launch");
    if (targets) {
        using O = MlpOffsets;
        float* g = reinterpret_cast<float*>(grad);
        ck(cudaMemsetAsync(g, 0, sizeof(float) * O::w1, stream), "cudaMemsetAsync(grad)");
        struct L { int in, out, w, b; } layers[4] = {
            {kMlpIn, kMlpHid, O::w1, O::b1}, {kMlpHid, kMlpHid, O::w2, O::b2},
            {kMlpHid, kMlpHid, O::w3, O::b3}, {kMlpHid, kMlpOut, O::w4, O::b4}};
        for (int l = 0; l < 4; ++l) {
            // kDwPadSmem bytes of unused dynamic shared memory hold an SM to
            // at most 6 of these CTAs (6 x 64 TMEM columns of 512), so no CTA
            // waits in tcgen05.alloc
            mlp_dw_kernel<<<chunks, kDwThreads, kDwPadSmem, stream>>>(bufs.act[l], bufs.dz[l], rows, layers[l].in,
                                                                      layers[l].out, part_w, part_b);
            ck(cudaGetLastError(), "mlp_dw_kernel launch");
            const int outs = layers[l].in * layers[l].out + layers[l].out;
            mlp_dw_reduce_kernel<<<(outs + 255) / 256, 256, 0, stream>>>(part_w, part_b, chunks, layers[l].in,
                                                                        layers[l].out, g + layers[l].w,
                                                                        g + layers[l].b);
            ck(cudaGetLastError(), "mlp_dw_reduce_kernel launch");
        }
        if (loss) {
            std::vector<double> part((size_t)blocks * kTrainWarps);
            ck(cudaMemcpyAsync(part.data(), bufs.sse, part.size() * sizeof(double), cudaMemcpyDeviceToHost, stream),
               "cudaMemcpyAsync(loss)");
            ck(cudaStreamSynchronize(stream), "cudaStreamSynchronize(loss)");
            double s = 0.0;
            for (double v : part) s += v;
            *loss = s / (3.0 * rows);
        }
    }
}

void mlp_adam(uintptr_t params, uintptr_t grad, uintptr_t m1, uintptr_t m2, float lr, int t, uintptr_t stream_u) {
    if (!params || !grad || !m1 || !m2) throw std::invalid_argument("mlp_adam: null device pointer");
    if (t < 1) throw std::invalid_argument("mlp_adam: step must be >= 1");
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f / (1.0f - std::pow(b1, (float)t)), c2 = 1.0f / (1.0f - std::pow(b2, (float)t));
    mlp_adam_kernel<<<16, 256, 0, reinterpret_cast<cudaStream_t>(stream_u)>>>(
        reinterpret_cast<float*>(params), reinterpret_cast<const float*>(grad), reinterpret_cast<float*>(m1),
        reinterpret_cast<float*>(m2), MlpOffsets::w1, MlpOffsets::total, lr, b1, b2, 1e-8f, c1, c2);
    ck(cudaGetLastError(), "mlp_adam_kernel launch");
}

// ---------------------------------------------------------------------------
// Allocation-free variant of mlp_gradients: its workspace is a fixed static
// device array of this file (one copy per device, allocated by the driver
// when the module loads), sized for kNoAllocMaxRows rows.
// ---------------------------------------------------------------------------
constexpr int kNoAllocMaxRows = CHYSX_MLP_NOALLOC_MAX_ROWS;
constexpr size_t align_up_c(size_t v) { return (v + kWsAlign - 1) / kWsAlign * kWsAlign; }
// loss partials of mlp_train_tile_kernel: one per warp of train_blocks(rows)
constexpr int kNoAllocPartials = (kNoAllocMaxRows + 16 * kTrainWarps - 1) / (16 * kTrainWarps) * kTrainWarps;
// the layout of mlp_workspace_bytes(kNoAllocMaxRows)
constexpr size_t kNoAllocScratchBytes =
    align_up_c(sizeof(MlpPacked)) + 8 * align_up_c((size_t)kNoAllocMaxRows * 64 * sizeof(__nv_bfloat16)) +
    align_up_c((size_t)kNoAllocPartials * sizeof(double)) +
    align_up_c((size_t)((kNoAllocMaxRows + kDwRows - 1) / kDwRows) * (64 * 64 + 64) * sizeof(float));
static_assert(kNoAllocPartials <= 1184 * kTrainWarps, "partials follow train_blocks()");

static __device__ __align__(256) unsigned char g_mlp_noalloc_scratch[kNoAllocScratchBytes];

unsigned char* g_noalloc_ptr[kMaxDevices] = {};

// Set-up, once per device and with that device current: the device address
// of this device's copy of the scratch array.  The lookup may load the
// module, so the first call on a device belongs before any stream capture.
unsigned char* noalloc_scratch() {
    const int dev = current_device();
    std::lock_guard<std::mutex> lock(g_dev_mu);
    if (!g_noalloc_ptr[dev]) {
        if (mlp_workspace_bytes(kNoAllocMaxRows) > kNoAllocScratchBytes)
            throw std::logic_error("chysx_mlp_gradients_noalloc: static scratch smaller than the workspace layout");
        void* p = nullptr;
        ck(cudaGetSymbolAddress(&p, g_mlp_noalloc_scratch), "cudaGetSymbolAddress(mlp scratch)");
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    }
    return g_noalloc_ptr[dev];
}

// mlp_gradients on the static scratch.  Nothing in the scratch must start at
// zero (every byte read is written earlier in the same call); the loss is
// summed on the host in the same order as mlp_gradients, from a stack copy of
// the per-warp partials.  Calls overlapping in time on one device race on the
// one scratch array.
void mlp_gradients_noalloc(uintptr_t params, uintptr_t features, uintptr_t targets, int rows, uintptr_t grad,
                           double* loss, uintptr_t stream_u) {
    if (rows <= 0) throw std::invalid_argument("chysx_mlp_gradients_noalloc: rows must be positive");
    if (rows > kNoAllocMaxRows)
        throw std::invalid_argument("chysx_mlp_gradients_noalloc: rows = " + std::to_string(rows) +
                                    " exceeds the static scratch limit of " + std::to_string(kNoAllocMaxRows) +
                                    " rows (CHYSX_MLP_NOALLOC_MAX_ROWS); use chysx_mlp_gradients with a workspace");
    if (!params || !features || !targets || !grad)
        throw std::invalid_argument("chysx_mlp_gradients_noalloc: null device pointer");
    unsigned char* ws = noalloc_scratch();
    mlp_gradients(params, features, targets, rows, grad, nullptr, 0, reinterpret_cast<uintptr_t>(ws),
                  kNoAllocScratchBytes, stream_u);
    if (loss) {
        auto stream = reinterpret_cast<cudaStream_t>(stream_u);
        const int n = train_blocks(rows) * kTrainWarps;
        // mlp_gradients' workspace layout: packed net, 8 row matrices, partials
        const size_t off = align_up(sizeof(MlpPacked)) + 8 * align_up((size_t)rows * 64 * sizeof(__nv_bfloat16));
        double part[kNoAllocPartials];
        ck(cudaMemcpyAsync(part, ws + off, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, stream),
           "cudaMemcpyAsync(loss)");
        ck(cudaStreamSynchronize(stream), "cudaStreamSynchronize(loss)");
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += part[i];
        *loss = s / (3.0 * rows);
    }
}

class ClothSim {
public:
    ~ClothSim() {
        destroy_graph();
        for (auto& e : ev_)
            if (e) cudaEventDestroy(e);
    }

    chysx_cloth_material mat{0.0f, 0.0f, 0.0f, 0.05f, 0.0f, 0.0f, 0.0f, -9.81f};

    // ---- caller buffers (borrowed) -------------------------------------
    void set_external_buffers(uintptr_t p, uintptr_t v, int count, uintptr_t w, uintptr_t f) {
        pos_ = p; vel_ = v; n_ = count; inv_mass_ = w; force_ = f;
    }

    // ---- mesh ----------------------------------------------------------
    void set_mesh(const int32_t* t, int T) {
        if (T < 0) throw std::invalid_argument("ClothSimulator::set_mesh: negative triangle count");
        if (T > 0 && !t) throw std::invalid_argument("ClothSimulator::set_mesh: null triangle array");
        tris_.assign(t, t + 3 * (size_t)T);
        // sorted unique undirected edges (src/cloth/cloth_simulator.cu:328-346)
        std::vector<long long> keys;
        keys.reserve(3 * (size_t)T);
        for (int q = 0; q < T; ++q) {
            const int v[3] = {t[3 * q], t[3 * q + 1], t[3 * q + 2]};
            for (int a = 0; a < 3; ++a) {
                const int x = v[a], y = v[(a + 1) % 3];
                const long long lo = std::min(x, y), hi = std::max(x, y);
                keys.push_back((lo << 32) | (unsigned long long)(unsigned)hi);
            }
        }
        std::sort(keys.begin(), keys.end());
        keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
        edges_.resize(2 * keys.size());
        for (size_t e = 0; e < keys.size(); ++e) {
            edges_[2 * e] = (int)(keys[e] >> 32);
            edges_[2 * e + 1] = (int)(unsigned)(keys[e] & 0xffffffffULL);
        }
        mesh_on_device_ = false;  // uploaded on first device use
        vt_n_ = -1;
        order_.clear();
        topo_dirty_ = true;
    }
    void ensure_mesh_on_device() {
        if (mesh_on_device_) return;
        d_tris_.upload(tris_);
        d_edges_.upload(edges_);
        mesh_on_device_ = true;
    }
    int num_edges() const { return (int)(edges_.size() / 2); }
    const std::vector<int>& edges() const { return edges_; }

    // ---- pins ----------------------------------------------------------
    void set_pins(const int32_t* idx, const float* tgt, int P, float k) {
        if (P < 0) throw std::invalid_argument("PinConstraint::set_pins: negative count");
        if (P > 0 && (!idx || !tgt)) throw std::invalid_argument("ClothSimulator::set_pins: null array");
        pin_idx_.assign(idx, idx + P);
        pin_tgt_.assign(tgt, tgt + 3 * (size_t)P);
        pin_k_ = k;
        topo_dirty_ = true;
    }
    void clear_pins() {
        pin_idx_.clear();
        pin_tgt_.clear();
        topo_dirty_ = true;
    }
    int num_pins() const { return (int)pin_idx_.size(); }

    // ---- static-shape contact (cloth_simulator.h:383-452) ---------------
    void add_static_plane(const float* nv, float d) {
        if (!nv) throw std::invalid_argument("ClothSimulator.add_static_plane: n must be a (3,) float32 vector");
        planes_.insert(planes_.end(), {nv[0], nv[1], nv[2], d});
        static_dirty_ = true;
    }
    void add_static_box(const float* c, const float* he, const float* ex, const float* ey, const float* ez) {
        for (const float* v : {c, he, ex, ey, ez})
            if (!v) throw std::invalid_argument("ClothSimulator.add_static_box: every argument is a (3,) vector");
        for (const float* v : {c, he, ex, ey, ez}) boxes_.insert(boxes_.end(), {v[0], v[1], v[2]});
        static_dirty_ = true;
    }
    void clear_static_shapes() {
        planes_.clear();
        boxes_.clear();
        static_dirty_ = true;
    }
    int static_planes() const { return (int)(planes_.size() / 4); }
    int static_boxes() const { return (int)(boxes_.size() / 15); }
    void set_static_param(int which, float v) {
        float* dst[4] = {&sc_thickness_, &sc_k_, &sc_mu_, &sc_eps_};
        if (*dst[which] != v) static_dirty_ = true;
        *dst[which] = v;
    }
    void get_static_params(float* t, float* k, float* mu, float* eps) const {
        if (t) *t = sc_thickness_;
        if (k) *k = sc_k_;
        if (mu) *mu = sc_mu_;
        if (eps) *eps = sc_eps_;
    }
    bool static_active() const { return sc_k_ > 0.0f && (!planes_.empty() || !boxes_.empty()); }

    // ---- contact operator (collision/contact_spmv.h:58-96) --------------
    void set_contact_op(const chysx_contact_op* op) {
        if (!op) throw std::invalid_argument("set_contact_op: null operator");
        // ContactSpMVOp::active (contact_spmv.h:88-92): an inactive op clears
        if (!(op->max_contacts > 0 && (op->stiffness > 0.0f || op->stiffnesses) && op->pairs)) {
            clear_contact_op();
            return;
        }
        if (!op->weights || !op->count)
            throw std::invalid_argument("set_contact_op: weights and count are required");
        if (op->max_contacts > (1 << 28)) throw std::invalid_argument("set_contact_op: max_contacts above 2^28");
        if ((op->pairs | op->weights | op->slips) & 15u)
            throw std::invalid_argument("set_contact_op: pairs, weights and slips must be 16-byte aligned");
        if ((op->count | op->stiffnesses) & 3u)
            throw std::invalid_argument("set_contact_op: count and stiffnesses must be 4-byte aligned");
        if (!(op->friction_mu >= 0.0f) || !(op->friction_epsilon > 0.0f))
            throw std::invalid_argument("set_contact_op: friction_mu >= 0 and friction_epsilon > 0 required");
        if (op->residual_mode != 0 && op->residual_mode != 1)
            throw std::invalid_argument("set_contact_op: residual_mode is 0 or 1");
        if (!co_active_ || !same_bytes(*op, co_)) graph_dirty_ = true;
        co_ = *op;
        co_active_ = true;
    }
    void clear_contact_op() {
        if (co_active_) graph_dirty_ = true;
        co_active_ = false;
        co_ = chysx_contact_op{};
    }
    void contact_stats(int* live, int* dropped, int* slots) {
        int st[4] = {0, 0, 0, 0};
        if (co_active_ && stepped_ && d_co_cnt_.size()) {
            ck(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(last_stream_)), "cudaStreamSynchronize");
            ck(cudaMemcpy(st, d_co_cnt_.get() + co_rows_ + 1, sizeof(st), cudaMemcpyDeviceToHost),
               "cudaMemcpy(contact stats)");
        }
        if (live) *live = st[0];
        if (dropped) *dropped = st[1];
        if (slots) *slots = st[2];
    }
    void update_pin_targets(const float* tgt, int P, uintptr_t stream) {
        if (!tgt || P <= 0) return;
        if (P != num_pins())
            throw std::invalid_argument(
                "ClothSimulator::update_pin_targets: n_pins does not match the currently installed pin "
                "set; call set_pins(...) to change the pin set instead.");
        std::memcpy(pin_tgt_.data(), tgt, 3 * (size_t)P * sizeof(float));
        if (!topo_dirty_ && (int)topo_.pin_perm.size() == P) {
            std::vector<float> sorted(3 * (size_t)P);
            for (int c = 0; c < P; ++c)
                for (int q = 0; q < 3; ++q) sorted[3 * c + q] = pin_tgt_[3 * (size_t)topo_.pin_perm[c] + q];
            // pageable source: returns once staged, ordered on `stream`
            ck(cudaMemcpyAsync(d_pin_tgt_.get(), sorted.data(), sorted.size() * sizeof(float),
                               cudaMemcpyHostToDevice, reinterpret_cast<cudaStream_t>(stream)),
               "cudaMemcpyAsync(pin targets)");
        }
    }

    // ---- springs / stretch ---------------------------------------------
    void build_springs(float k, const float* k_per_edge, uintptr_t stream) {
        const int E = num_edges();
        springs_built_ = true;
        topo_dirty_ = true;
        if (E == 0) {
            d_rest_.reset();
            d_kedge_.reset();
            return;
        }
        if (!pos_)
            throw std::runtime_error(
                "ClothSimulator::build_springs_from_current_positions: external positions must be set "
                "first via set_external_buffers().");
        check_indices(edges_, "spring edge");
        ensure_mesh_on_device();
        std::vector<float> ke(E, k);
        if (k_per_edge) std::memcpy(ke.data(), k_per_edge, E * sizeof(float));
        d_kedge_.upload(ke);
        d_rest_.resize(E);
        rest_length_kernel<<<grid_for(E, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
            d_edges_.get(), reinterpret_cast<const float*>(pos_), d_rest_.get(), E);
        ck(cudaGetLastError(), "rest_length_kernel launch");
    }
    int num_springs() const { return springs_built_ ? num_edges() : 0; }

    void build_stretch(float k, const float* k_per_tri, uintptr_t stream) {
        const int T = (int)(tris_.size() / 3);
        stretch_built_ = true;
        topo_dirty_ = true;
        if (T == 0) {
            d_dminv_.reset();
            d_area_.reset();
            d_ktri_.reset();
            return;
        }
        if (!pos_)
            throw std::runtime_error(
                "ClothSimulator::build_fem_stretch_from_current_positions: external positions must be "
                "set first via set_external_buffers().");
        check_indices(tris_, "triangle");
        ensure_mesh_on_device();
        std::vector<float> kt(T, k);
        if (k_per_tri) std::memcpy(kt.data(), k_per_tri, T * sizeof(float));
        d_ktri_.upload(kt);
        d_dminv_.resize(T);
        d_area_.resize(T);
        rest_shape_kernel<<<grid_for(T, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
            d_tris_.get(), reinterpret_cast<const float*>(pos_), d_dminv_.get(), d_area_.get(), T,
            det_eps_, 1.0f, 0.0f);
        ck(cudaGetLastError(), "rest_shape_kernel launch");
    }

    // ClothSimulator::build_fem_shear_from_current_positions
    // (cloth_simulator.cu:423-449): the stretch element over the same
    // triangles with its rest frame turned by pi/4, a second (Dm^-1, area,
    // k) set assembled beside the stretch set.
    void build_shear(float k, const float* k_per_tri, uintptr_t stream) {
        const int T = (int)(tris_.size() / 3);
        shear_built_ = true;
        topo_dirty_ = true;
        if (T == 0) {
            d_dminv_s_.reset();
            d_area_s_.reset();
            d_ktri_s_.reset();
            return;
        }
        if (!pos_)
            throw std::runtime_error(
                "ClothSimulator::build_fem_shear_from_current_positions: external positions must be "
                "set first via set_external_buffers().");
        check_indices(tris_, "triangle");
        ensure_mesh_on_device();
        std::vector<float> kt(T, k);
        if (k_per_tri) std::memcpy(kt.data(), k_per_tri, T * sizeof(float));
        d_ktri_s_.upload(kt);
        d_dminv_s_.resize(T);
        d_area_s_.resize(T);
        const float quarter_pi = 0.7853981633974483f;
        rest_shape_kernel<<<grid_for(T, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
            d_tris_.get(), reinterpret_cast<const float*>(pos_), d_dminv_s_.get(), d_area_s_.get(), T,
            det_eps_, std::cos(quarter_pi), std::sin(quarter_pi));
        ck(cudaGetLastError(), "rest_shape_kernel launch (shear)");
    }

    // ClothSimulator::build_bending_from_current_positions
    // (cloth_simulator.cu:451-514): dihedrals of the current mesh, rest
    // angles from the current positions, one stiffness for all.
    void build_bending(float k, uintptr_t stream) {
        bending_built_ = true;
        k_bend_ = k;
        topo_dirty_ = true;
        if (tris_.empty()) {
            dih_.clear();
            d_dih_.reset();
            d_rest_angle_.reset();
            return;
        }
        if (!pos_)
            throw std::runtime_error(
                "ClothSimulator::build_bending_from_current_positions: external positions must be set "
                "first via set_external_buffers().");
        check_indices(tris_, "triangle");
        build_dihedrals(tris_, dih_);
        const int D = (int)(dih_.size() / 4);
        if (D == 0) {
            d_dih_.reset();
            d_rest_angle_.reset();
            return;
        }
        std::vector<int4> hd(D);
        for (int d = 0; d < D; ++d) hd[d] = make_int4(dih_[4 * d], dih_[4 * d + 1], dih_[4 * d + 2], dih_[4 * d + 3]);
        d_dih_.upload(hd);
        d_rest_angle_.resize(D);
        bending_rest_kernel<<<grid_for(D, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
            d_dih_.get(), reinterpret_cast<const float*>(pos_), d_rest_angle_.get(), D);
        ck(cudaGetLastError(), "bending_rest_kernel launch");
    }
    int num_dihedrals() const { return bending_built_ ? (int)(dih_.size() / 4) : 0; }

    // ---- mass ----------------------------------------------------------
    void redistribute_mass(float rho, uintptr_t inv_mass, int count, uintptr_t stream) {
        if (count <= 0) return;
        if (!inv_mass)
            throw std::invalid_argument(
                "ClothSimulator::redistribute_mass_area_weighted: inv_mass_ptr must be non-null");
        if (rho <= 0.0f)
            throw std::invalid_argument(
                "ClothSimulator::redistribute_mass_area_weighted: surface_density must be positive");
        if (tris_.empty())
            throw std::runtime_error(
                "ClothSimulator::redistribute_mass_area_weighted: call set_mesh(...) before "
                "redistributing mass.");
        if (!pos_ || n_ < count)
            throw std::runtime_error(
                "ClothSimulator::redistribute_mass_area_weighted: external positions must be set first "
                "via set_external_buffers().");
        ensure_mesh_on_device();
        if (vt_n_ != count) {
            std::vector<int> off, list;
            build_vertex_triangles(count, tris_, off, list);
            d_vt_off_.upload(off);
            d_vt_list_.upload(list);
            vt_n_ = count;
        }
        lumped_inv_mass_kernel<<<grid_for(count, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
            d_vt_off_.get(), d_vt_list_.get(), d_tris_.get(), reinterpret_cast<const float*>(pos_),
            rho / 3.0f, reinterpret_cast<float*>(inv_mass), count);
        ck(cudaGetLastError(), "lumped_inv_mass_kernel launch");
    }

    // ---- solver --------------------------------------------------------
    void set_pcg_iterations(int m) {
        if (m < 0 || m > 10000000)
            throw std::invalid_argument("set_pcg_iterations: max_iter must be in [0, 1e7]");
        max_iter_ = m;
    }
    int pcg_iterations() const { return max_iter_; }
    void set_solver(int m, double tol, int warm) {
        if (m < 0 || m > 10000000) throw std::invalid_argument("set_solver: max_iter must be in [0, 1e7]");
        if (!(tol >= 0.0) || !std::isfinite(tol)) throw std::invalid_argument("set_solver: rel_tol must be >= 0");
        if (warm < CHYSX_WARM_ZERO || warm > CHYSX_WARM_PREVIOUS_SCALED)
            throw std::invalid_argument("set_solver: unknown warm_start mode");
        if (warm == CHYSX_WARM_LEARNED && !warm_guess_)
            throw std::runtime_error("set_solver: learned warm start needs a network (load one first)");
        if (warm != warm_mode_) graph_dirty_ = true;
        max_iter_ = m;
        rel_tol_ = tol;
        warm_mode_ = warm;
    }
    void set_options(int sis, int af, float eps) {
        if (!(eps >= 0.0f)) throw std::invalid_argument("set_options: fem_det_eps must be >= 0");
        if ((sis != 0) != springs_in_step_) topo_dirty_ = true;
        springs_in_step_ = sis != 0;
        apply_force_ = af != 0;
        det_eps_ = eps;
    }

    // ---- step ----------------------------------------------------------
    void step(float dt, uintptr_t stream) {
        if (n_ <= 0) return;
        if (!pos_ || !vel_)
            throw std::runtime_error(
                "chysx::cloth::ClothSimulator::step: pos / vel spans must be set via "
                "set_external_buffers() before stepping.");
        if (!(dt > 0.0f)) throw std::invalid_argument("chysx::cloth::ClothSimulator::step: dt must be positive");
        ensure_mesh_on_device();
        if (topo_dirty_ || topo_.n_ext != n_) rebuild_topology();
        if (co_active_ && !inst_offsets_.empty())
            throw std::invalid_argument("the contact operator needs the single-instance layout");
        if (static_dirty_) {
            std::vector<float> sh(planes_);
            sh.insert(sh.end(), boxes_.begin(), boxes_.end());
            d_shapes_.upload(sh);
            static_dirty_ = false;
            graph_dirty_ = true;
        }
        if (graph_dirty_) build_graph();
        update_step_nodes(dt);
        ck(cudaGraphLaunch(exec_, reinterpret_cast<cudaStream_t>(stream)), "cudaGraphLaunch(step)");
        last_stream_ = stream;
        stepped_ = true;
    }

    // One step from (pos_in, vel_in) into (pos_out, vel_out): the double-
    // buffered stepping of a host that keeps state_in and state_out (the
    // reference's Newton bridge copies state_in to state_out and steps that
    // in place, README.md:113-130); the inputs become the external buffers.
    void step_into(float dt, uintptr_t pin, uintptr_t vin, uintptr_t pout, uintptr_t vout, uintptr_t stream) {
        if (!pin || !vin || !pout || !vout) throw std::invalid_argument("step_into: null state buffer");
        const uintptr_t bytes = (uintptr_t)n_ * 12u;
        auto overlap = [&](uintptr_t a, uintptr_t b) { return a != b && a < b + bytes && b < a + bytes; };
        if (overlap(pin, pout) || overlap(vin, vout) || overlap(pin, vout) || overlap(vin, pout) ||
            (pout != pin && (pout == vin || vout == pin)) || pout == vout)
            throw std::invalid_argument("step_into: output buffers must equal or not overlap the inputs");
        if ((pout == pin) != (vout == vin))
            throw std::invalid_argument("step_into: step both or neither of pos / vel in place");
        pos_ = pin;
        vel_ = vin;
        pos_out_ = pout;
        vel_out_ = vout;
        struct Reset {
            ClothSim* s;
            ~Reset() { s->pos_out_ = s->vel_out_ = 0; }
        } reset{this};
        step(dt, stream);
    }

    void last_stats(int* iters, double* relres, int* status) {
        int it = 0, st = 0;
        double rr = 0.0, bb = 0.0;
        if (stepped_) {
            ck(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(last_stream_)), "cudaStreamSynchronize");
            if (graph_path_ == kPathPersistent) {
                // a batch reports its slowest / worst instance
                std::vector<InstState> s(plan_.n_inst);
                ck(cudaMemcpy(s.data(), d_inst_.get(), s.size() * sizeof(InstState), cudaMemcpyDeviceToHost),
                   "cudaMemcpy(state)");
                double worst = -1.0;
                for (const InstState& q : s) {
                    it = std::max(it, q.iter);
                    st = std::max(st, q.status);
                    const double rel = q.bb > 0.0 ? std::max(q.rr, 0.0) / q.bb : 0.0;
                    if (rel > worst) { worst = rel; rr = q.rr; bb = q.bb; }
                }
            } else {
                SolveState s{};
                ck(cudaMemcpy(&s, d_state_.get(), sizeof(SolveState), cudaMemcpyDeviceToHost), "cudaMemcpy(state)");
                it = s.iter; st = s.status; rr = s.rr; bb = s.bb;
            }
        }
        if (iters) *iters = it;
        if (relres) *relres = (bb > 0.0) ? std::sqrt(std::max(rr, 0.0) / bb) : 0.0;
        if (status) *status = st;
    }

    // True residual of the returned iterate (pcg_solver.h:78,191): when on,
    // every step also computes ||b - (A + C) dx|| / ||b|| from the stored
    // system and the final dx, per instance.
    void set_true_residual(int on) {
        if ((on != 0) != true_res_) graph_dirty_ = true;
        true_res_ = on != 0;
    }
    // per-instance true relative residuals of the last step (n = instances);
    // worst = the largest.  Needs set_true_residual(1) before that step.
    void true_residual(int n, double* rel, double* worst) {
        if (!true_res_ || !stepped_ || d_tres_.size() == 0)
            throw std::runtime_error("true_residual: enable it with set_true_residual(1) before the step");
        const int ni = (int)topo_.inst_slice.size() - 1;
        if (rel && n != ni) throw std::invalid_argument("true_residual: wrong instance count");
        ck(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(last_stream_)), "cudaStreamSynchronize");
        std::vector<double2> h(d_tres_.size());
        ck(cudaMemcpy(h.data(), d_tres_.get(), h.size() * sizeof(double2), cudaMemcpyDeviceToHost),
           "cudaMemcpy(true residual)");
        double w = 0.0;
        for (int b = 0; b < ni; ++b) {
            double rr = 0.0, bb = 0.0;
            for (int sl = topo_.inst_slice[b]; sl < topo_.inst_slice[b + 1]; ++sl) {
                rr += h[sl].x;
                bb += h[sl].y;
            }
            const double q = bb > 0.0 ? std::sqrt(rr / bb) : 0.0;
            if (rel) rel[b] = q;
            w = std::max(w, q);
        }
        if (worst) *worst = w;
    }

    // Learned warm start: loads a network (flat FP32 parameters, MlpOffsets).
    void set_network(const float* params, int n) {
        if (n != MlpOffsets::total)
            throw std::invalid_argument("set_network: expected " + std::to_string(MlpOffsets::total) + " parameters");
        if (!params) throw std::invalid_argument("set_network: null parameters");
        for (int q = 0; q < n; ++q)
            if (!std::isfinite(params[q])) throw std::invalid_argument("set_network: non-finite parameter");
        d_net_params_.upload(params, n);
        d_net_.resize(1);
        mlp_pack_kernel<<<8, 256>>>(d_net_params_.get(), d_net_.get());
        ck(cudaGetLastError(), "mlp_pack_kernel launch");
        ck(cudaDeviceSynchronize(), "cudaDeviceSynchronize(set_network)");
        warm_guess_ = true;
        graph_dirty_ = true;
    }
    // Exports each step's raw per-particle features (n x 20 floats, caller
    // order) to a device buffer; 0 disables.
    void set_feature_output(uintptr_t ptr, uintptr_t pred) {
        if ((ptr != 0) != (feat_out_ != 0)) graph_dirty_ = true;
        feat_out_ = ptr;
        pred_out_ = ptr ? pred : 0;
        nodes_valid_ = false;  // node arguments changed
    }
    // instances whose solve kept the warm-start guess in the last step
    int guess_kept() {
        if (!stepped_ || graph_path_ != kPathPersistent) return 0;
        ck(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(last_stream_)), "cudaStreamSynchronize");
        std::vector<InstState> s(plan_.n_inst);
        ck(cudaMemcpy(s.data(), d_inst_.get(), s.size() * sizeof(InstState), cudaMemcpyDeviceToHost),
           "cudaMemcpy(instance states)");
        if (warm_mode_ == CHYSX_WARM_ZERO) return 0;
        int kept = 0;
        for (const InstState& q : s) kept += q.fallback ? 0 : 1;
        return kept;
    }
    bool want_features() const { return warm_mode_ == CHYSX_WARM_LEARNED || feat_out_ != 0; }
    // warm argument of the solver kernels: 0 zero guess, 1 guess as given
    // (the reference's previous dx), 2 energy-scaled guess
    int warm_kernel_mode() const {
        if (warm_mode_ == CHYSX_WARM_ZERO) return 0;
        return warm_mode_ == CHYSX_WARM_PREVIOUS ? 1 : 2;
    }

    // Declares independent cloth instances: particles [off[b], off[b+1]).
    void set_instances(const int32_t* off, int n_inst) {
        if (n_inst < 0) throw std::invalid_argument("set_instances: negative instance count");
        if (n_inst > 0 && !off) throw std::invalid_argument("set_instances: null offsets");
        if (n_inst == 0) inst_offsets_.clear();
        else inst_offsets_.assign(off, off + n_inst + 1);
        order_.clear();
        topo_dirty_ = true;
    }
    // Row order (no counterpart in the reference): 0 = the caller's particle
    // order (default), 1 = spatially compact blocks (recursive coordinate
    // bisection of the positions at the next topology build, kept until the
    // mesh, the instances or the particle count change), so that the rows a
    // CTA holds form a patch of the cloth.
    void set_row_order(int mode) {
        if (mode != 0 && mode != 1) throw std::invalid_argument("set_row_order: mode must be 0 or 1");
        if (mode != row_order_) {
            order_.clear();
            topo_dirty_ = true;
        }
        row_order_ = mode;
    }
    int row_order() const { return row_order_; }
    // internal row of every particle (identity without a mapped layout)
    void row_of_particles(int n, int32_t* out) const {
        if (n != topo_.n_ext) throw std::invalid_argument("row_of_particles: wrong particle count");
        for (int e = 0; e < n; ++e) out[e] = topo_.ext_to_row.empty() ? e : topo_.ext_to_row[e];
    }
    int num_instances() const { return inst_offsets_.empty() ? 1 : (int)inst_offsets_.size() - 1; }
    void instance_stats(int n, int* iters, double* relres, int* status) {
        if (!stepped_ || graph_path_ != kPathPersistent)
            throw std::runtime_error("instance_stats: needs a step taken with the persistent solver");
        if (n != plan_.n_inst) throw std::invalid_argument("instance_stats: wrong instance count");
        ck(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(last_stream_)), "cudaStreamSynchronize");
        std::vector<InstState> s(n);
        ck(cudaMemcpy(s.data(), d_inst_.get(), s.size() * sizeof(InstState), cudaMemcpyDeviceToHost),
           "cudaMemcpy(instance states)");
        for (int b = 0; b < n; ++b) {
            if (iters) iters[b] = s[b].iter;
            if (relres) relres[b] = s[b].bb > 0.0 ? std::sqrt(std::max(s[b].rr, 0.0) / s[b].bb) : 0.0;
            if (status) status[b] = s[b].status;
        }
    }

    // Solver kernel selection (no counterpart in the reference): path 0 =
    // persistent cooperative PCG (register-resident rows when the system is
    // small enough, else streamed), 1 = graph WHILE loop of two kernels,
    // 2 = streamed persistent kernel forced.  block / grid of the streamed
    // persistent kernel (0 = automatic).
    // Synchronisation of the persistent kernels: 0 = grid-wide counter
    // barrier (default), 1 = per-instance polled reduction slots.
    void set_sync(int mode) {
        if (mode < 0 || mode > 1) throw std::invalid_argument("set_sync_mode: mode must be 0 or 1");
        if (mode != sync_mode_) graph_dirty_ = true;
        sync_mode_ = mode;
    }
    int sync_mode() const { return sync_mode_; }
    void set_tuning(int path, int block, int grid) {
        if (path < 0 || path > 2) throw std::invalid_argument("set_tuning: path must be 0, 1 or 2");
        if (block != 0 && block != 128 && block != 256 && block != 512)
            throw std::invalid_argument("set_tuning: block must be 0, 128, 256 or 512");
        if (grid < 0) throw std::invalid_argument("set_tuning: grid must be >= 0");
        solver_path_ = path;
        pcg_block_ = block ? block : 256;
        pcg_block_req_ = block;
        pcg_grid_req_ = grid;
        graph_dirty_ = true;
    }
    // Preconditioner (no counterpart in the reference, whose PCG is
    // block-Jacobi): 0 = block-Jacobi (default), 1 = CTA-local Chebyshev of
    // odd degree on [lambda_max / ratio, lambda_max], 2 = that plus a coarse
    // level of one rigid translation per CTA block (single-instance plans of
    // at most kCoarseMaxBlocks CTAs; otherwise it acts as 1); used by the
    // register-resident kernel, the others stay block-Jacobi.
    void set_preconditioner(int kind, int degree, float ratio) {
        if (kind < 0 || kind > 2) throw std::invalid_argument("set_preconditioner: kind must be 0, 1 or 2");
        if (kind >= 1 && (degree < 1 || degree > 63 || degree % 2 == 0))
            throw std::invalid_argument("set_preconditioner: degree must be odd, 1 to 63");
        if (kind >= 1 && !(ratio > 1.0f && ratio < 1.0e6f))
            throw std::invalid_argument("set_preconditioner: ratio must be in (1, 1e6)");
        if (kind != pc_kind_) graph_dirty_ = true;
        pc_kind_ = kind;
        pc_degree_ = kind ? degree : 0;
        pc_ratio_ = kind ? ratio : 0.0f;
    }
    void preconditioner(int* kind, int* degree, float* ratio, int* in_use) const {
        if (kind) *kind = pc_kind_;
        if (degree) *degree = pc_degree_;
        if (ratio) *ratio = pc_ratio_;
        if (in_use) *in_use = coarse_on_ ? (coarse_nq_ > 1 ? 3 : 2) : (pc_active() ? 1 : 0);
    }
    // the CTA-local preconditioner runs in the register-resident kernel of
    // the default synchronisation mode (with the coarse level where the plan
    // is a single instance)
    bool pc_active() const { return pc_kind_ >= 1 && resident_ && graph_path_ == kPathPersistent && sync_mode_ == 0; }

    // kernel actually used by the last graph build: 0 resident, 1 loop,
    // 2 streamed
    void solver_info(int* path, int* grid, int* block) const {
        const int used = graph_path_ == kPathLoop ? 1 : (resident_ ? 0 : 2);
        if (path) *path = used;
        if (grid) *grid = used == 1 ? 0 : plan_.grid;
        if (block) *block = used == 1 ? kVecBlock : (resident_ ? resident_warps_ * 32 : pcg_block_);
    }

    // ---- autotuner (no counterpart in the reference) -------------------
    // Times the solver configurations that apply to the current system on
    // the current state and keeps the fastest one.  Candidates: the resident
    // / streamed persistent kernel picked by the planner (rows per CTA and
    // CTAs per SM follow from it), the streamed kernel at 128 / 256 / 512
    // threads (4 / 8 / 16 slices, i.e. rows x 32, per CTA), each with both
    // synchronisation modes, and
    // the graph-loop path.  Every trial solves the same system: the caller's
    // positions / velocities and the previous-step guess are restored before
    // each trial and at the end, so the simulation does not advance.
    struct TuneResult {
        int path, block, sync;            // the candidate (set_tuning / sync values)
        int used, used_grid, used_block;  // what the planner launched (solver_info)
        int iters, status;
        float solve_ms;                   // best of the repetitions
    };
    const std::vector<TuneResult>& tune_results() const { return tune_; }

    void autotune(float dt, int reps, uintptr_t stream_u) {
        if (n_ <= 0 || !pos_ || !vel_) throw std::runtime_error("autotune: set_external_buffers() first");
        if (!(dt > 0.0f)) throw std::invalid_argument("autotune: dt must be positive");
        if (reps < 1 || reps > 100) throw std::invalid_argument("autotune: reps must be in [1, 100]");
        auto stream = reinterpret_cast<cudaStream_t>(stream_u);
        ensure_mesh_on_device();
        if (topo_dirty_ || topo_.n_ext != n_) rebuild_topology();
        const size_t nb = 12 * (size_t)n_;
        DevBuf<float> save_pos, save_vel;
        DevBuf<float4> save_x;
        save_pos.resize(3 * (size_t)n_);
        save_vel.resize(3 * (size_t)n_);
        save_x.resize(d_x_.size());
        ck(cudaMemcpyAsync(save_pos.get(), reinterpret_cast<void*>(pos_), nb, cudaMemcpyDeviceToDevice, stream),
           "autotune: save positions");
        ck(cudaMemcpyAsync(save_vel.get(), reinterpret_cast<void*>(vel_), nb, cudaMemcpyDeviceToDevice, stream),
           "autotune: save velocities");
        if (d_x_.size())
            ck(cudaMemcpyAsync(save_x.get(), d_x_.get(), d_x_.size() * sizeof(float4), cudaMemcpyDeviceToDevice,
                               stream), "autotune: save guess");
        auto restore = [&] {
            ck(cudaMemcpyAsync(reinterpret_cast<void*>(pos_), save_pos.get(), nb, cudaMemcpyDeviceToDevice, stream),
               "autotune: restore positions");
            ck(cudaMemcpyAsync(reinterpret_cast<void*>(vel_), save_vel.get(), nb, cudaMemcpyDeviceToDevice, stream),
               "autotune: restore velocities");
            if (save_x.size())
                ck(cudaMemcpyAsync(d_x_.get(), save_x.get(), save_x.size() * sizeof(float4), cudaMemcpyDeviceToDevice,
                                   stream), "autotune: restore guess");
        };
        const bool timing0 = timing_;
        enable_timing(1);
        struct Cand { int path, block, sync; };
        std::vector<Cand> cands;
        for (int sync : {0, 1}) {
            cands.push_back({kPathPersistent, 256, sync});
            for (int block : {128, 256, 512}) cands.push_back({kPathStreamed, block, sync});
        }
        if (topo_.inst_slice.size() <= 2) cands.push_back({kPathLoop, 256, 0});
        tune_.clear();
        for (const Cand& c : cands) {
            solver_path_ = c.path;
            pcg_block_ = c.block;
            pcg_block_req_ = c.block;
            pcg_grid_req_ = 0;
            sync_mode_ = c.sync;
            graph_dirty_ = true;
            TuneResult r{c.path, c.block, c.sync, 0, 0, 0, 0, 0, 1e30f};
            for (int k = 0; k < reps; ++k) {
                restore();
                step(dt, stream_u);
                float a = 0.f, sm = 0.f, f = 0.f;
                last_timing(&a, &sm, &f);
                double rr = 0.0;
                last_stats(&r.iters, &rr, &r.status);
                r.solve_ms = std::min(r.solve_ms, sm);
            }
            solver_info(&r.used, &r.used_grid, &r.used_block);
            // the planner may turn a candidate into one already timed
            bool dup = false;
            for (const TuneResult& q : tune_)
                dup |= q.used == r.used && q.used_grid == r.used_grid && q.used_block == r.used_block &&
                       q.sync == r.sync;
            if (!dup) tune_.push_back(r);
        }
        const TuneResult* best = nullptr;
        for (const TuneResult& q : tune_)
            if (q.status != kSolveNonfinite && q.status != kSolveKernelError && (!best || q.solve_ms < best->solve_ms))
                best = &q;
        if (!best) throw std::runtime_error("autotune: no configuration solved the system");
        solver_path_ = best->path;
        pcg_block_ = best->block;
        pcg_block_req_ = best->block;
        pcg_grid_req_ = 0;
        sync_mode_ = best->sync;
        graph_dirty_ = true;
        restore();
        ck(cudaStreamSynchronize(stream), "autotune: synchronise");
        enable_timing(timing0 ? 1 : 0);
    }

    // Optional event-record nodes around the graph's phases (measurement only).
    void enable_timing(int on) {
        if ((on != 0) != timing_) graph_dirty_ = true;
        timing_ = on != 0;
        if (timing_ && !ev_[0])
            for (auto& e : ev_) ck(cudaEventCreate(&e), "cudaEventCreate");
    }
    void last_timing(float* assemble_ms, float* solve_ms, float* finalize_ms) {
        if (!timing_ || !stepped_ || !ev_[0]) throw std::runtime_error("timing is not enabled");
        ck(cudaEventSynchronize(ev_[3]), "cudaEventSynchronize");
        float a = 0.f, b = 0.f, c = 0.f;
        ck(cudaEventElapsedTime(&a, ev_[0], ev_[1]), "cudaEventElapsedTime");
        ck(cudaEventElapsedTime(&b, ev_[1], ev_[2]), "cudaEventElapsedTime");
        ck(cudaEventElapsedTime(&c, ev_[2], ev_[3]), "cudaEventElapsedTime");
        if (assemble_ms) *assemble_ms = a;
        if (solve_ms) *solve_ms = b;
        if (finalize_ms) *finalize_ms = c;
    }

    int num_particles() const { return n_; }
    int num_off_diag_blocks() const { return (int)topo_.nnz(); }

    // The coarse level of the last step (test support): info = {on, coarse
    // blocks, CTAs per block, fields per block, unknowns m, band half-width};
    // with ac / ainv non-null (m x m floats each, cap >= m * m) A_c dense and
    // the rows of A_c^-1 the CTAs computed, unknown B U + 3 q + c.
    void debug_coarse(int32_t* info, float* ac, float* ainv, int cap) {
        ck(cudaDeviceSynchronize(), "debug_coarse sync");
        const int U = 3 * coarse_nq_, m = coarse_on_ ? U * coarse_nb_ : 0;
        if (info) {
            info[0] = coarse_on_ ? 1 : 0;
            info[1] = coarse_nb_;
            info[2] = coarse_g_;
            info[3] = coarse_nq_;
            info[4] = m;
            info[5] = 0;  // no band: A_c is inverted densely
        }
        if (!coarse_on_ || (!ac && !ainv)) return;
        if (cap < m * m) throw std::invalid_argument("debug_coarse: cap below m * m");
        if (ac) {
            const int mn = coarse_mn_;
            std::vector<float> blocks((size_t)coarse_nb_ * mn * U * U);
            std::vector<int> nbr((size_t)coarse_nb_ * mn), cnt(coarse_nb_);
            ck(cudaMemcpy(blocks.data(), d_cac_.get(), blocks.size() * sizeof(float), cudaMemcpyDeviceToHost), "copy A_c");
            ck(cudaMemcpy(nbr.data(), d_cnbr_.get(), nbr.size() * sizeof(int), cudaMemcpyDeviceToHost), "copy lists");
            ck(cudaMemcpy(cnt.data(), d_ccnt_.get(), cnt.size() * sizeof(int), cudaMemcpyDeviceToHost), "copy counts");
            std::fill(ac, ac + (size_t)m * m, 0.0f);
            for (int B = 0; B < coarse_nb_; ++B)
                for (int k = 0; k < cnt[B]; ++k) {
                    const int C = nbr[(size_t)B * mn + k];
                    const float* b = blocks.data() + ((size_t)B * mn + k) * U * U;
                    for (int r = 0; r < U; ++r)
                        for (int c = 0; c < U; ++c) ac[(size_t)(B * U + r) * m + C * U + c] = b[r * U + c];
                }
        }
        if (ainv && coarse_batched_) {
            // the batched level's inverse, block-diagonal by instance
            const int ni = plan_.n_inst;
            std::vector<int> ib(ni + 1), ao(ni + 1);
            ck(cudaMemcpy(ib.data(), d_inst_blk_.get(), ib.size() * sizeof(int), cudaMemcpyDeviceToHost), "copy blocks");
            ck(cudaMemcpy(ao.data(), d_inst_aoff_.get(), ao.size() * sizeof(int), cudaMemcpyDeviceToHost), "copy offsets");
            std::vector<float> inv((size_t)std::max(1, ao[ni]));
            ck(cudaMemcpy(inv.data(), d_cainv_.get(), (size_t)ao[ni] * sizeof(float), cudaMemcpyDeviceToHost),
               "copy A_c^-1 blocks");
            std::fill(ainv, ainv + (size_t)m * m, 0.0f);
            for (int b = 0; b < ni; ++b) {
                const int o = U * ib[b], mb = U * (ib[b + 1] - ib[b]);
                for (int r = 0; r < mb; ++r)
                    for (int c = 0; c < mb; ++c) ainv[(size_t)(o + r) * m + o + c] = inv[(size_t)ao[b] + (size_t)r * mb + c];
            }
        } else if (ainv) {
            ck(cudaMemcpy(ainv, d_cainv_.get(), (size_t)m * m * sizeof(float), cudaMemcpyDeviceToHost), "copy A_c^-1");
        }
    }
    // The coarse blocks' first internal rows (nb + 1 entries, the last the
    // row count rounded to slices); returns nb + 1 (0 without a coarse level).
    int debug_coarse_rows(int32_t* row0, int cap) {
        if (!coarse_on_) return 0;
        const int n = coarse_nb_ + 1;
        if (row0) {
            if (cap < n) throw std::invalid_argument("debug_coarse_rows: cap below the block count + 1");
            ck(cudaMemcpy(row0, d_cb_row0_.get(), (size_t)n * sizeof(int), cudaMemcpyDeviceToHost), "copy block rows");
        }
        return n;
    }
    void debug_dump(float* diag, int32_t* rp, int32_t* col, float* vals, float* rhs, float* dx) {
        const int n = topo_.n_ext;
        if (n == 0 || topo_.n == 0) return;
        ck(cudaDeviceSynchronize(), "cudaDeviceSynchronize(debug_dump)");
        const size_t np = topo_.n_pad;
        std::vector<float> hd(np * 6), hv(d_val_.size());
        std::vector<float4> hb(np), hx(np);
        ck(cudaMemcpy(hd.data(), d_diag_.get(), hd.size() * 4, cudaMemcpyDeviceToHost), "dump diag");
        if (!hv.empty()) ck(cudaMemcpy(hv.data(), d_val_.get(), hv.size() * 4, cudaMemcpyDeviceToHost), "dump val");
        ck(cudaMemcpy(hb.data(), d_b_.get(), np * sizeof(float4), cudaMemcpyDeviceToHost), "dump rhs");
        ck(cudaMemcpy(hx.data(), d_x_.get(), np * sizeof(float4), cudaMemcpyDeviceToHost), "dump dx");
        auto put9 = [](float* o, const float* s6) {
            const float xx = s6[0], xy = s6[32], xz = s6[64], yy = s6[96], yz = s6[128], zz = s6[160];
            o[0] = xx; o[1] = xy; o[2] = xz; o[3] = xy; o[4] = yy; o[5] = yz; o[6] = xz; o[7] = yz; o[8] = zz;
        };
        const int ow = off_width();
        const bool mapped = !topo_.ext_to_row.empty();
        int k_out = 0;
        if (rp) rp[0] = 0;
        for (int e = 0; e < n; ++e) {
            const int r = mapped ? topo_.ext_to_row[e] : e;
            if (diag) put9(diag + 9 * (size_t)e, &hd[(size_t)(r >> 5) * 192 + (r & 31)]);
            if (rhs) { rhs[3 * e] = hb[r].x; rhs[3 * e + 1] = hb[r].y; rhs[3 * e + 2] = hb[r].z; }
            if (dx) { dx[3 * e] = hx[r].x; dx[3 * e + 1] = hx[r].y; dx[3 * e + 2] = hx[r].z; }
            const int so = topo_.slice_off[r >> 5];
            // the row's entries by particle index (the reference's CSR order),
            // whatever order the internal rows are in
            std::vector<std::pair<int, int>> ent;
            for (int q = topo_.csr_ptr[r]; q < topo_.csr_ptr[r + 1]; ++q)
                ent.emplace_back(mapped ? topo_.row_to_ext[topo_.csr_col[q]] : topo_.csr_col[q], q);
            std::sort(ent.begin(), ent.end());
            for (const auto& cq : ent) {
                const int q = cq.second;
                if (col) col[k_out] = cq.first;
                if (vals) {
                    const int el = topo_.csr_to_ell[q];
                    const float* src = &hv[(size_t)so * ow + (size_t)((el - so) >> 5) * ow * 32 + (el & 31)];
                    if (ow == 6) put9(vals + 9 * (size_t)k_out, src);
                    else
                        for (int c = 0; c < 9; ++c) vals[9 * (size_t)k_out + c] = src[c * 32];
                }
                ++k_out;
            }
            if (rp) rp[e + 1] = k_out;
        }
    }

    // learned warm start hook (set by the network module)
    bool warm_guess_ = false;

private:
    void check_indices(const std::vector<int>& idx, const char* what) const {
        for (int v : idx)
            if (v < 0 || v >= n_)
                throw std::out_of_range(std::string(what) + " vertex index " + std::to_string(v) +
                                        " out of range [0, " + std::to_string(n_) + ")");
    }

    void rebuild_topology() {
        const bool use_stretch = stretch_built_ && d_dminv_.size() > 0;
        const bool use_shear = shear_built_ && d_dminv_s_.size() > 0;
        const bool use_tris = use_stretch || use_shear;
        const bool use_bending = bending_built_ && d_dih_.size() > 0;
        const bool use_springs = springs_built_ && springs_in_step_ && d_rest_.size() > 0;
        if (!inst_offsets_.empty() && inst_offsets_.back() != n_)
            throw std::invalid_argument("set_instances: offsets do not cover the particle count");
        if (row_order_ == 1 && (int)order_.size() != n_) {
            // positions at this build order the rows for the rest of the run
            std::vector<float> hp(3 * (size_t)n_);
            if (n_ > 0)
                ck(cudaMemcpy(hp.data(), reinterpret_cast<const void*>(pos_), hp.size() * sizeof(float),
                              cudaMemcpyDeviceToHost),
                   "cudaMemcpy(positions for the row order)");
            spatial_order(hp.data(), n_, inst_offsets_, order_);
        }
        const std::vector<int> no_order;
        build_topology(n_, tris_, use_tris, edges_, use_springs, pin_idx_, inst_offsets_, topo_, dih_, use_bending,
                       row_order_ == 1 ? order_ : no_order);
        if (topo_.row_to_ext.empty()) d_row_to_ext_.reset();
        else d_row_to_ext_.upload(topo_.row_to_ext);
        if (topo_.ext_to_row.empty()) d_ext_to_row_.reset();
        else d_ext_to_row_.upload(topo_.ext_to_row);
        use_tris_ = use_tris;
        use_stretch_ = use_stretch;
        use_shear_ = use_shear;
        use_springs_ = use_springs;
        use_bending_ = use_bending;
        d_slice_off_.upload(topo_.slice_off);
        d_col_.upload(topo_.col);
        d_val_.resize(std::max<size_t>(1, (size_t)topo_.ell_entries() * off_width()));
        d_val_.zero();
        d_diag_.resize((size_t)topo_.n_pad * 6);
        d_dnl_.resize((size_t)topo_.n_pad * 6);
        d_minv_.resize((size_t)topo_.n_pad * 6);
        d_tinc_off_.upload(topo_.tinc_off);
        d_tinc_.upload(topo_.tinc);
        d_tinc_meta_.upload(topo_.tinc_meta);
        d_sinc_off_.upload(topo_.sinc_off);
        d_sinc_.upload(topo_.sinc);
        d_sinc_meta_.upload(topo_.sinc_meta);
        d_dinc_off_.upload(topo_.dinc_off);
        d_dinc_.upload(topo_.dinc);
        d_dinc_meta_.upload(topo_.dinc_meta);
        d_pin_off_.upload(topo_.pin_off);
        d_pin_row_.upload(topo_.pin_row);
        {
            std::vector<float> sorted(3 * topo_.pin_row.size());
            for (size_t c = 0; c < topo_.pin_row.size(); ++c)
                for (int q = 0; q < 3; ++q) sorted[3 * c + q] = pin_tgt_[3 * (size_t)topo_.pin_perm[c] + q];
            d_pin_tgt_.upload(sorted);
        }
        const size_t np = topo_.n_pad;
        if (d_x_.size() != np) {
            // a resize starts the warm-start history from zero
            // (src/cloth/cloth_simulator.cu:802-811)
            for (DevBuf<float4>* b : {&d_b_, &d_r_, &d_z_, &d_x_, &d_ap_, &d_p0_, &d_p1_}) {
                b->resize(np);
                b->zero();
            }
        }
        // assembly block size: per-thread shared accumulators of
        // (6 or 9) * width floats
        const int W = std::max(1, topo_.max_width);
        asm_block_ = (W * off_width() <= 96) ? 128 : (W * off_width() <= 192 ? 64 : 32);
        asm_smem_ = (size_t)off_width() * W * asm_block_ * sizeof(double);
        if (asm_smem_ > kMaxAssembleSmem)
            throw std::runtime_error("a row has " + std::to_string(W) +
                                     " neighbours, more than the assembly's FP64 row accumulators hold (" +
                                     std::to_string(kMaxAssembleSmem / (sizeof(double) * 32 * off_width())) + ")");
        const int max_grid = std::max(grid_for(topo_.n, asm_block_), grid_for(topo_.n, kVecBlock));
        d_part_.resize((size_t)std::max(1, max_grid) * 7);
        d_state_.resize(1);
        d_state_.zero();
        topo_dirty_ = false;
        graph_dirty_ = true;
    }

    DevTopo dev_topo() const {
        DevTopo t;
        t.n = topo_.n;
        t.n_slices = topo_.n_slices;
        t.slice_off = d_slice_off_.get();
        t.col = d_col_.get();
        t.val = d_val_.get();
        t.diag = d_diag_.get();
        t.dnl = d_dnl_.get();
        t.minv = d_minv_.get();
        t.tinc_off = d_tinc_off_.get();
        t.tinc = d_tinc_.get();
        t.tinc_meta = d_tinc_meta_.get();
        t.sinc_off = d_sinc_off_.get();
        t.sinc = d_sinc_.get();
        t.sinc_meta = d_sinc_meta_.get();
        t.pin_off = d_pin_off_.get();
        t.pin_row = d_pin_row_.get();
        t.pin_tgt = d_pin_tgt_.get();
        t.dinc_off = d_dinc_off_.get();
        t.dinc = d_dinc_.get();
        t.dinc_meta = d_dinc_meta_.get();
        t.nsym = use_bending_ ? 1 : 0;
        t.co.off = d_co_off_.get();
        t.co.ent = d_co_ent_.get();
        t.co.rec = d_co_rec_.get();
        t.co.active = co_active_ ? 1 : 0;
        t.co.residual = co_.residual_mode == 0 ? 1 : 0;
        return t;
    }
    ElemData elem_data() const {
        ElemData e;
        e.tris = d_tris_.get();
        e.dminv = d_dminv_.get();
        e.area = d_area_.get();
        e.ktri = d_ktri_.get();
        e.dminv_s = d_dminv_s_.get();
        e.area_s = d_area_s_.get();
        e.ktri_s = d_ktri_s_.get();
        e.edges = d_edges_.get();
        e.rest = d_rest_.get();
        e.kedge = d_kedge_.get();
        e.pin_k = pin_k_;
        e.use_tris = use_tris_ ? 1 : 0;
        e.use_stretch = use_stretch_ ? 1 : 0;
        e.use_shear = use_shear_ ? 1 : 0;
        e.dih = d_dih_.get();
        e.rest_angle = d_rest_angle_.get();
        e.k_bend = k_bend_;
        e.use_bending = use_bending_ ? 1 : 0;
        e.use_springs = use_springs_ ? 1 : 0;
        e.sc.shapes = d_shapes_.get();
        e.sc.n_planes = static_planes();
        e.sc.n_boxes = static_boxes();
        e.sc.thickness = sc_thickness_;
        e.sc.k = sc_k_;
        e.sc.mu = sc_mu_;
        e.sc.eps = sc_eps_;
        e.sc.active = static_active() ? 1 : 0;
        return e;
    }
    Vecs vecs() const {
        return Vecs{d_b_.get(), d_r_.get(), d_z_.get(), d_x_.get(), d_ap_.get(), d_p0_.get(), d_p1_.get()};
    }
    StepArgs step_args(float dt) const {
        StepArgs a;
        a.pos = reinterpret_cast<float*>(pos_);
        a.vel = reinterpret_cast<float*>(vel_);
        a.pos_out = reinterpret_cast<float*>(pos_out_ ? pos_out_ : pos_);
        a.vel_out = reinterpret_cast<float*>(vel_out_ ? vel_out_ : vel_);
        a.inv_mass = reinterpret_cast<const float*>(inv_mass_);
        a.force = reinterpret_cast<const float*>(force_);
        a.row_to_ext = d_row_to_ext_.get();
        a.n = topo_.n;
        a.dt = dt;
        a.gx = mat.gx; a.gy = mat.gy; a.gz = mat.gz;
        a.damping = mat.damping;
        a.apply_force = apply_force_ ? 1 : 0;
        a.want_features = want_features() ? 1 : 0;
        return a;
    }
    SolverCfg solver_cfg() const {
        SolverCfg c;
        std::memset(&c, 0, sizeof(c));  // compared bytewise
        c.max_iter = max_iter_;
        c.use_tol = rel_tol_ > 0.0 ? 1 : 0;
        c.rel_tol = rel_tol_;
        c.pc_degree = pc_kind_ >= 1 ? pc_degree_ : 0;
        c.pc_ratio = pc_kind_ >= 1 ? pc_ratio_ : 0.0f;
        return c;
    }

    // the graph-loop path needs the build that sets the WHILE condition
    const void* assemble_fn() const {
        const bool loop = solver_path_ == kPathLoop;
        if (asm_block_ == 128)
            return loop ? reinterpret_cast<const void*>(&assemble_kernel<128, 1>)
                        : reinterpret_cast<const void*>(&assemble_kernel<128, 0>);
        if (asm_block_ == 64)
            return loop ? reinterpret_cast<const void*>(&assemble_kernel<64, 1>)
                        : reinterpret_cast<const void*>(&assemble_kernel<64, 0>);
        return loop ? reinterpret_cast<const void*>(&assemble_kernel<32, 1>)
                    : reinterpret_cast<const void*>(&assemble_kernel<32, 0>);
    }

    void asm_params(cudaKernelNodeParams& p, void** args) {
        p = cudaKernelNodeParams{};
        p.func = const_cast<void*>(assemble_fn());
        p.gridDim = dim3(grid_for(topo_.n, asm_block_));
        p.blockDim = dim3(asm_block_);
        p.sharedMemBytes = (unsigned)asm_smem_;
        p.kernelParams = args;
    }

    void destroy_graph() {
        if (exec_) cudaGraphExecDestroy(exec_);
        if (graph_) cudaGraphDestroy(graph_);
        exec_ = nullptr;
        graph_ = nullptr;
        cfield_node_ = nullptr;
    }

    void build_graph() {
        if (solver_path_ == kPathLoop && topo_.inst_slice.size() > 2)
            throw std::invalid_argument("the graph-loop solver path solves a single instance; use path 0 or 2");
        if (solver_path_ == kPathLoop) build_graph_loop();
        else build_graph_persistent();
    }

    void guess_params(cudaKernelNodeParams& p, void** args) const {
        p = cudaKernelNodeParams{};
        p.func = reinterpret_cast<void*>(&learned_guess_kernel);
        const int tiles = std::max(1, (topo_.n + kGuessThreads - 1) / kGuessThreads);
        p.gridDim = dim3(std::max(1, std::min(2048, tiles)));
        p.blockDim = dim3(kGuessThreads);
        p.kernelParams = args;
    }
    // Appends the feature / learned-guess node after `dep` when needed.
    cudaGraphNode_t add_guess_node(cudaGraphNode_t dep, StepArgs& a, DevTopo& t, Vecs& v) {
        guess_node_ = nullptr;
        if (!want_features()) return dep;
        const MlpPacked* net = d_net_.get();
        float* fo = reinterpret_cast<float*>(feat_out_);
        float* po = reinterpret_cast<float*>(pred_out_);
        int predict = warm_mode_ == CHYSX_WARM_LEARNED ? 1 : 0;
        void* args[] = {&a, &t, &v, &net, &fo, &po, &predict};
        cudaKernelNodeParams p;
        guess_params(p, args);
        ck(cudaGraphAddKernelNode(&guess_node_, graph_, &dep, 1, &p), "add learned-guess node");
        return guess_node_;
    }
    void patch_guess_node(StepArgs& a, DevTopo& t, Vecs& v) {
        if (!guess_node_) return;
        const MlpPacked* net = d_net_.get();
        float* fo = reinterpret_cast<float*>(feat_out_);
        float* po = reinterpret_cast<float*>(pred_out_);
        int predict = warm_mode_ == CHYSX_WARM_LEARNED ? 1 : 0;
        void* args[] = {&a, &t, &v, &net, &fo, &po, &predict};
        cudaKernelNodeParams p;
        guess_params(p, args);
        ck(cudaGraphExecKernelNodeSetParams(exec_, guess_node_, &p), "update learned-guess node");
    }

    // Appends an event-record node after `dep` when timing is on.
    cudaGraphNode_t timing_node(int k, cudaGraphNode_t dep) {
        if (!timing_) return dep;
        cudaGraphNode_t node;
        ck(cudaGraphAddEventRecordNode(&node, graph_, dep ? &dep : nullptr, dep ? 1 : 0, ev_[k]),
           "cudaGraphAddEventRecordNode");
        return node;
    }

    static constexpr int kResidentMaxWidth = 8;
    template <int SYNC>
    const void* persistent_fn_sync() const {
        if (resident_) {
            // rows of a triangulated grid have at most 6 off-diagonal blocks;
            // the 6-wide build fits a row in 128 registers with fewer spills
            // (ptxas: 56 B of spill stores, the 8-wide build 128 B)
            if (coarse_on_ && SYNC == 0) {
                if (topo_.max_width <= 6)
                    return resident_warps_ == 16 ? reinterpret_cast<const void*>(&pcg_resident_kernel<16, 6, 0, 2>)
                                                 : reinterpret_cast<const void*>(&pcg_resident_kernel<8, 6, 0, 2>);
                return resident_warps_ == 16
                           ? reinterpret_cast<const void*>(&pcg_resident_kernel<16, kResidentMaxWidth, 0, 2>)
                           : reinterpret_cast<const void*>(&pcg_resident_kernel<8, kResidentMaxWidth, 0, 2>);
            }
            if (pc_kind_ >= 1 && SYNC == 0) {
                if (topo_.max_width <= 6)
                    return resident_warps_ == 16 ? reinterpret_cast<const void*>(&pcg_resident_kernel<16, 6, 0, 1>)
                                                 : reinterpret_cast<const void*>(&pcg_resident_kernel<8, 6, 0, 1>);
                return resident_warps_ == 16
                           ? reinterpret_cast<const void*>(&pcg_resident_kernel<16, kResidentMaxWidth, 0, 1>)
                           : reinterpret_cast<const void*>(&pcg_resident_kernel<8, kResidentMaxWidth, 0, 1>);
            }
            if (topo_.max_width <= 6)
                return resident_warps_ == 16 ? reinterpret_cast<const void*>(&pcg_resident_kernel<16, 6, SYNC>)
                                             : reinterpret_cast<const void*>(&pcg_resident_kernel<8, 6, SYNC>);
            return resident_warps_ == 16
                       ? reinterpret_cast<const void*>(&pcg_resident_kernel<16, kResidentMaxWidth, SYNC>)
                       : reinterpret_cast<const void*>(&pcg_resident_kernel<8, kResidentMaxWidth, SYNC>);
        }
        if (pcg_block_ == 64) {
            // the planner's choice for batches with the coarse level only (synchronisation mode 0)
            if (SYNC != 0) throw std::logic_error("64-thread streamed kernel without synchronisation mode 0");
            if (coarse_on_ && coarse_batched_) return reinterpret_cast<const void*>(&pcg_persistent_kernel<64, 0, 2>);
            return reinterpret_cast<const void*>(&pcg_persistent_kernel<64, 0, 0>);
        }
        if (coarse_on_ && SYNC == 0 && coarse_batched_) {
            if (pcg_block_ == 128) return reinterpret_cast<const void*>(&pcg_persistent_kernel<128, 0, 2>);
            if (pcg_block_ == 512) return reinterpret_cast<const void*>(&pcg_persistent_kernel<512, 0, 2>);
            return reinterpret_cast<const void*>(&pcg_persistent_kernel<256, 0, 2>);
        }
        if (coarse_on_ && SYNC == 0) {
            if (pcg_block_ == 128) return reinterpret_cast<const void*>(&pcg_persistent_kernel<128, 0, 1>);
            if (pcg_block_ == 512) return reinterpret_cast<const void*>(&pcg_persistent_kernel<512, 0, 1>);
            return reinterpret_cast<const void*>(&pcg_persistent_kernel<256, 0, 1>);
        }
        if (pcg_block_ == 128) return reinterpret_cast<const void*>(&pcg_persistent_kernel<128, SYNC>);
        if (pcg_block_ == 512) return reinterpret_cast<const void*>(&pcg_persistent_kernel<512, SYNC>);
        return reinterpret_cast<const void*>(&pcg_persistent_kernel<256, SYNC>);
    }
    const void* persistent_fn() const { return sync_mode_ ? persistent_fn_sync<1>() : persistent_fn_sync<0>(); }

    // neighbour-exchange buffer k of the resident kernels (null otherwise)
    void* exchange_buffer(int k) const {
        const size_t np = (size_t)std::max(1, topo_.n_pad);
        if (resident_) return d_zp_.get() + k * np;
        return nullptr;
    }

    BatchPlan batch_plan() const {
        BatchPlan bp;
        bp.n_inst = plan_.n_inst;
        bp.max_slices_per_cta = plan_.max_slices_per_cta;
        bp.max_inst_per_cta = plan_.max_inst_per_cta;
        bp.slice_inst = d_slice_inst_.get();
        bp.inst_slice = d_inst_slice_.get();
        bp.cta_slice = d_cta_slice_.get();
        bp.cta_inst_lo = d_cta_inst_lo_.get();
        bp.cta_inst_hi = d_cta_inst_hi_.get();
        bp.inst_cta_lo = d_inst_cta_lo_.get();
        bp.inst_slot = d_inst_slot_.get();
        bp.slots = d_slots_.get();
        bp.inst = d_inst_.get();
        bp.bar = d_bar_.get();
        bp.n_slots = plan_.inst_slot.empty() ? 0 : plan_.inst_slot.back();
        bp.fslots = sync_mode_ ? d_fslots_.get() : nullptr;
        bp.cg = coarse_on_ ? d_cargs_.get() : nullptr;
        return bp;
    }

    // Plans the persistent launch: as many co-resident CTAs as useful, one
    // warp per slice at least.
    // Register-resident plan: one slice per warp, W warps per CTA, all CTAs
    // co-resident.  Returns false when the system does not fit.
    bool plan_resident(int sms) {
        resident_ = false;  // a previous plan's choice must not leak into this one
        // the register-resident rows hold symmetric blocks only
        // (and have no contact-operator gather)
        if (solver_path_ != kPathPersistent || topo_.max_width > kResidentMaxWidth || use_bending_ || co_active_)
            return false;
        const int n_slices = std::max(1, topo_.n_slices);
        for (int W : {16, 8}) {
            resident_ = true;
            resident_warps_ = W;
            const int grid = (n_slices + W - 1) / W;
            build_plan(topo_.inst_slice, grid, plan_);
            plan_coarse();
            pers_smem_ = (size_t)W * kSlotW * sizeof(double) + (size_t)plan_.max_inst_per_cta * sizeof(LocalInst);
            if (coarse_on_)  // the coarse block's rows of A_c^-1, a phase's block values and its staged slots
                pers_smem_ += ((size_t)9 * coarse_nq_ * coarse_nq_ * coarse_nb_ + (size_t)3 * coarse_nq_ * coarse_nb_) *
                                  sizeof(float) + 16 + (size_t)plan_.inst_slot.back() * kSlotW * sizeof(double) + 16;
            // static + dynamic above 48 KB needs the opt-in
            ck(cudaFuncSetAttribute(persistent_fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pers_smem_),
               "cudaFuncSetAttribute(resident smem)");
            int per_sm = 0;
            ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_fn(), W * 32, pers_smem_),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor(resident)");
            if (per_sm >= 1 && plan_.grid <= per_sm * sms && plan_.max_slices_per_cta <= W) return true;
        }
        resident_ = false;
        return false;
    }

    // Coarse level of the two-level preconditioner (kind 2) of a
    // single-instance resident plan: coarse blocks of G consecutive CTAs with
    // nq fields each; (G, nq) = (kCoarseResidentCtas, 4) (translation and
    // linear fields on 2-CTA blocks) where the plan has at least 8 CTAs and
    // the coarse system at most kCoarseDenseMax unknowns, else (1, 1) (the
    // translation of every CTA block).  The streamed kernel's blocks are larger (about
    // kCoarseStreamRows rows).  Host side:
    // the coarse block of every slice and its first row, every block's sorted
    // list of the blocks its rows touch, and the list position of every ELL
    // entry's column block.
    // The coarse blocks' neighbour lists (every block a coarse row of A_c
    // touches, itself included, sorted), the list position of every ELL
    // entry's column block, and the block layout, uploaded; false (nothing
    // uploaded) when a block touches more than kCoarseMaxNbr blocks.
    bool coarse_neighbours(const std::vector<int>& slice_cb, const std::vector<int>& row0, int nb, int& mn) {
        std::vector<std::vector<int>> lists(nb);
        for (int B = 0; B < nb; ++B) {
            std::vector<int>& l = lists[B];
            l.push_back(B);
            for (int sl = row0[B] / 32; sl < row0[B + 1] / 32; ++sl)
                for (int e = topo_.slice_off[sl]; e < topo_.slice_off[sl + 1]; ++e) l.push_back(slice_cb[topo_.col[e] >> 5]);
            std::sort(l.begin(), l.end());
            l.erase(std::unique(l.begin(), l.end()), l.end());
            if ((int)l.size() > kCoarseMaxNbr) return false;
        }
        mn = 1;
        for (const auto& l : lists) mn = std::max(mn, (int)l.size());
        std::vector<int> nbr((size_t)nb * mn, -1), cnt(nb), self(nb);
        for (int B = 0; B < nb; ++B) {
            cnt[B] = (int)lists[B].size();
            for (int k = 0; k < cnt[B]; ++k) {
                nbr[(size_t)B * mn + k] = lists[B][k];
                if (lists[B][k] == B) self[B] = k;
            }
        }
        std::vector<unsigned char> ell(std::max<size_t>(1, topo_.col.size()), 0);
        for (int B = 0; B < nb; ++B)
            for (int sl = row0[B] / 32; sl < row0[B + 1] / 32; ++sl)
                for (int e = topo_.slice_off[sl]; e < topo_.slice_off[sl + 1]; ++e) {
                    const int cb = slice_cb[topo_.col[e] >> 5];
                    ell[e] = (unsigned char)(std::lower_bound(lists[B].begin(), lists[B].end(), cb) - lists[B].begin());
                }
        d_slice_cb_.upload(slice_cb);
        d_cb_row0_.upload(row0);
        d_cnbr_.upload(nbr);
        d_ccnt_.upload(cnt);
        d_cself_.upload(self);
        d_ell_nbr_.upload(ell);
        return true;
    }
    bool plan_coarse_with(int G, int nq, double shift) {
        const int grid = plan_.grid, ns = topo_.n_slices;
        const int nb = (grid + G - 1) / G, U = 3 * nq, m = U * nb;
        if (m > kCoarseDenseMax) return false;
        std::vector<int> slice_cb(std::max(1, ns), 0), row0(nb + 1, 0);
        for (int c = 0; c < grid; ++c)
            for (int sl = plan_.cta_slice[c]; sl < plan_.cta_slice[c + 1]; ++sl) slice_cb[sl] = c / G;
        for (int B = 0; B <= nb; ++B) row0[B] = plan_.cta_slice[std::min(grid, B * G)] * 32;
        int mn = 0;
        if (!coarse_neighbours(slice_cb, row0, nb, mn)) return false;
        if (nq > 1) {
            d_cw_.resize((size_t)std::max(1, row0[nb]));
            d_cw_.zero();
        }
        d_cac_.resize((size_t)nb * mn * U * U);
        d_cac_.zero();
        // split every block's slices over CTAs of ~kCoarseSplitSlices slices
        int spb = 1;
        for (int B = 0; B < nb; ++B) spb = std::max(spb, (row0[B + 1] - row0[B] + 31) / 32);
        const int splits = std::min(kCoarseMaxSplits, std::max(1, (spb + kCoarseSplitSlices - 1) / kCoarseSplitSlices));
        d_cacp_.resize((size_t)splits * nb * mn * U * U);
        d_cainv_.resize((size_t)m * m);
        d_cainv_.zero();
        {
            const size_t mp = (size_t)(m + 31) / 32 * 32;  // kInvTile padding
            d_cwork_.resize(mp * mp + mp + 2 * 32 * 32);
            d_cfail_.resize(1);
            d_cfail_.zero();
            d_cbar_.resize(1);
            d_cbar_.zero();
        }
        coarse_shift_ = shift;
        coarse_nb_ = nb;
        coarse_mn_ = mn;
        coarse_splits_ = splits;
        coarse_g_ = G;
        coarse_nq_ = nq;
        coarse_on_ = true;
        const CoarseArgs cargs = coarse_args();
        d_cargs_.upload(&cargs, 1);
        ck(cudaFuncSetAttribute(reinterpret_cast<const void*>(&coarse_assemble_kernel),
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coarse_assemble_smem()),
           "cudaFuncSetAttribute(coarse assemble smem)");
        return true;
    }
    void plan_coarse() {
        coarse_on_ = false;
        coarse_batched_ = false;
        if (pc_kind_ != 2 || sync_mode_ != 0) return;
        if (plan_.n_inst != 1) {
            // several instances on the streamed kernel, zero-guess solves:
            // one coarse block per instance
            if (!resident_ && warm_mode_ == CHYSX_WARM_ZERO && !plan_coarse_batched(kBatchMaxBlocks))
                plan_coarse_batched(1);
            return;
        }
        if (!resident_) {
            // streamed kernel: coarse blocks of G CTAs, about
            // kCoarseStreamRows rows each, translation and linear fields,
            // A_c inverted densely (at most kCoarseDenseMax unknowns)
            const int rows_per_cta = std::max(1, 32 * topo_.n_slices / std::max(1, plan_.grid));
            int G = std::max(1, (kCoarseStreamRows + rows_per_cta / 2) / rows_per_cta);
            while (G <= plan_.grid) {
                const int nb = (plan_.grid + G - 1) / G;
                if (nb >= 2 && plan_coarse_with(G, 4, kCoarseShift)) return;
                if (nb < 2) return;
                ++G;
            }
            return;
        }
        if (plan_.grid > kCoarseMaxBlocks) return;
        if (plan_.grid >= 8 && plan_coarse_with(kCoarseResidentCtas, 4, 0.0)) return;
        plan_coarse_with(1, 1, 0.0);
    }
    // The batched coarse level of the streamed kernel: coarse blocks inside
    // instances, each a run of G_b consecutive segment slots of instance b
    // (a segment: the instance's rows in one CTA), G_b the least that keeps
    // at most kBatchMaxBlocks blocks per instance; translation and linear
    // fields (12 unknowns) per block.  Blocks couple inside their instance
    // only, so A_c is block-diagonal by instance and each instance's dense
    // inverse (at most 144 unknowns) is formed on its own
    // (coarse_invert_batched_kernel).  With max_blocks = 1: one block per
    // instance.
    bool plan_coarse_batched(int max_blocks) {
        const int ni = plan_.n_inst, ns = topo_.n_slices, nq = 4, U = 3 * nq;
        const int n_slots = plan_.inst_slot.back();
        std::vector<int> blk_slot{0}, inst_blk(ni + 1, 0), inst_aoff(ni + 1, 0), slot_cb(std::max(1, n_slots), 0);
        int mmax = U;
        for (int b = 0; b < ni; ++b) {
            const int lo = plan_.inst_slot[b], hi = plan_.inst_slot[b + 1];
            const int G = std::max(1, (hi - lo + max_blocks - 1) / max_blocks);
            for (int k = lo; k < hi; k += G) {
                const int B = (int)blk_slot.size() - 1, k1 = std::min(hi, k + G);
                for (int kk = k; kk < k1; ++kk) slot_cb[kk] = B;
                blk_slot.push_back(k1);
            }
            inst_blk[b + 1] = (int)blk_slot.size() - 1;
            const int m = U * (inst_blk[b + 1] - inst_blk[b]);
            mmax = std::max(mmax, m);
            inst_aoff[b + 1] = inst_aoff[b] + m * m;
        }
        const int nb = (int)blk_slot.size() - 1;
        // a block's rows: from the first slice of its first segment (slot k of
        // instance b is CTA inst_cta_lo[b] + k - inst_slot[b]) to the next block's
        std::vector<int> row0(nb + 1, ns * 32), slice_cb(std::max(1, ns), 0);
        for (int b = 0; b < ni; ++b)
            for (int B = inst_blk[b]; B < inst_blk[b + 1]; ++B) {
                const int c = plan_.inst_cta_lo[b] + blk_slot[B] - plan_.inst_slot[b];
                row0[B] = std::max(plan_.cta_slice[c], plan_.inst_slice[b]) * 32;
            }
        for (int B = 0; B < nb; ++B)
            for (int sl = row0[B] / 32; sl < row0[B + 1] / 32; ++sl) slice_cb[sl] = B;
        int mn = 0;
        if (!coarse_neighbours(slice_cb, row0, nb, mn)) return false;
        d_blk_slot_.upload(blk_slot);
        d_inst_blk_.upload(inst_blk);
        d_inst_aoff_.upload(inst_aoff);
        d_slot_cb_.upload(slot_cb);
        d_cw_.resize((size_t)std::max(1, row0[nb]));
        d_cw_.zero();
        d_cac_.resize((size_t)nb * mn * U * U);
        d_cac_.zero();
        int spb = 1;
        for (int B = 0; B < nb; ++B) spb = std::max(spb, (row0[B + 1] - row0[B] + 31) / 32);
        const int splits = std::min(kCoarseMaxSplits, std::max(1, (spb + kCoarseSplitSlices - 1) / kCoarseSplitSlices));
        d_cacp_.resize((size_t)splits * nb * mn * U * U);
        d_cainv_.resize((size_t)std::max(1, inst_aoff[ni]));
        d_cainv_.zero();
        d_cfail_.resize(1);
        d_cfail_.zero();
        d_cbar_.resize(1);
        d_cbar_.zero();
        coarse_shift_ = kCoarseShift;
        coarse_nb_ = nb;
        coarse_mn_ = mn;
        coarse_splits_ = splits;
        coarse_g_ = 1;
        coarse_nq_ = nq;
        coarse_on_ = true;
        coarse_batched_ = true;
        batched_mmax_ = mmax;
        const CoarseArgs cargs = coarse_args();
        d_cargs_.upload(&cargs, 1);
        ck(cudaFuncSetAttribute(reinterpret_cast<const void*>(&coarse_assemble_kernel),
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coarse_assemble_smem()),
           "cudaFuncSetAttribute(coarse assemble smem)");
        ck(cudaFuncSetAttribute(reinterpret_cast<const void*>(&coarse_invert_batched_kernel),
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)batched_invert_smem(mmax)),
           "cudaFuncSetAttribute(batched coarse inverse smem)");
        return true;
    }
    // the streamed kernel's shared memory for its coarse level: the block
    // values (dense level) or the per-instance values (batched level)
    size_t coarse_stream_smem() const {
        if (!coarse_on_) return 0;
        if (coarse_batched_) return (size_t)plan_.max_inst_per_cta * kInstCoarseW * sizeof(float) + 16;
        return (size_t)3 * coarse_nq_ * coarse_nb_ * sizeof(float) + 16;
    }
    // per-lane partial sums of the coarse assembly: [nq][9][max_nbr][32] floats
    size_t coarse_assemble_smem() const {
        return (size_t)coarse_nq_ * 9 * coarse_mn_ * 32 * sizeof(float);
    }
    CoarseArgs coarse_args() const {
        CoarseArgs c{};
        c.on = coarse_on_ ? 1 : 0;
        c.nb = coarse_nb_;
        c.g = coarse_g_;
        c.nq = coarse_nq_;
        c.m = 3 * coarse_nq_ * coarse_nb_;
        c.max_nbr = coarse_mn_;
        c.slice_cb = d_slice_cb_.get();
        c.cb_row0 = d_cb_row0_.get();
        c.nbr = d_cnbr_.get();
        c.nbr_cnt = d_ccnt_.get();
        c.self_idx = d_cself_.get();
        c.ell_nbr = d_ell_nbr_.get();
        c.w = coarse_nq_ > 1 ? d_cw_.get() : nullptr;
        c.ac = d_cac_.get();
        c.acp = d_cacp_.get();
        c.splits = coarse_splits_;
        c.ainv = d_cainv_.get();
        c.dense = resident_ || coarse_batched_ ? 0 : 1;
        c.batched = coarse_batched_ ? 1 : 0;
        c.blk_slot = coarse_batched_ ? d_blk_slot_.get() : nullptr;
        c.inst_blk = coarse_batched_ ? d_inst_blk_.get() : nullptr;
        c.inst_aoff = coarse_batched_ ? d_inst_aoff_.get() : nullptr;
        c.slot_cb = coarse_batched_ ? d_slot_cb_.get() : nullptr;
        c.shift = coarse_shift_;
        c.work = d_cwork_.get();
        c.fail = d_cfail_.get();
        return c;
    }

    void plan_persistent() {
        int dev = 0, sms = 0;
        ck(cudaGetDevice(&dev), "cudaGetDevice");
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
        if (plan_resident(sms)) {
            upload_plan();
            d_zp_.resize(2 * (size_t)std::max(1, topo_.n_pad));
            d_zp_.zero();
            return;
        }
        if (pcg_block_req_ == 0) {
            // batches with the coarse level inside instances: CTAs of 128
            // threads, twice as many segments and so coarse blocks (batch512:
            // 6.05 against 5.10 steps/s, 526 against 632 iterations per step,
            // the same time per iteration); otherwise 256
            const bool batched_coarse = pc_kind_ == 2 && sync_mode_ == 0 && warm_mode_ == CHYSX_WARM_ZERO &&
                                        topo_.inst_slice.size() > 2;
            pcg_block_ = batched_coarse ? 64 : 256;
        }
        const int W = pcg_block_ / 32;
        const int n_slices = std::max(1, topo_.n_slices);
        // shared memory depends on the plan; iterate once with a generous bound
        int grid = pcg_grid_req_ > 0 ? pcg_grid_req_ : std::max(1, (n_slices + W - 1) / W);
        for (int pass = 0; pass < 3; ++pass) {
            build_plan(topo_.inst_slice, grid, plan_);
            pers_smem_ = (size_t)plan_.max_slices_per_cta * kSlotW * sizeof(double) +
                         (size_t)plan_.max_inst_per_cta * sizeof(LocalInst);
            // static + dynamic above 48 KB needs the opt-in
            ck(cudaFuncSetAttribute(persistent_fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pers_smem_),
               "cudaFuncSetAttribute(persistent smem)");
            int per_sm = 0;
            ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_fn(), pcg_block_, pers_smem_),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
            if (per_sm < 1) throw std::runtime_error("persistent PCG kernel cannot be resident (shared memory)");
            const int cap = per_sm * sms;
            if (plan_.grid <= cap) break;
            grid = cap;
        }
        plan_coarse();
        if (coarse_on_) {
            // the coarse block values (or the batched level's per-instance values) behind the records
            const size_t extra = coarse_stream_smem();
            pers_smem_ += extra;
            ck(cudaFuncSetAttribute(persistent_fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pers_smem_),
               "cudaFuncSetAttribute(persistent smem)");
            int per_sm = 0;
            ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_fn(), pcg_block_, pers_smem_),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
            if (per_sm * sms < plan_.grid) {
                coarse_on_ = false;  // the extra shared memory costs co-residency: plain block-Jacobi
                coarse_batched_ = false;
                pers_smem_ -= extra;
            }
        }
        upload_plan();
    }

    // Host-side invariants of the persistent launch, checked before any
    // launch: the kernel's shared-memory layout fits the bytes requested and
    // the resident kernel owns at most one slice per warp.
    void check_plan() const {
        const size_t li_bytes = (size_t)plan_.max_inst_per_cta * sizeof(LocalInst);
        size_t need = resident_ ? (size_t)resident_warps_ * kSlotW * sizeof(double) + li_bytes
                                : (size_t)plan_.max_slices_per_cta * kSlotW * sizeof(double) + li_bytes;
        if (!resident_) need += coarse_stream_smem();
        if (pers_smem_ < need || (resident_ && plan_.max_slices_per_cta > resident_warps_) ||
            (!resident_ && pcg_block_ / 32 < 1))
            throw std::logic_error("persistent PCG plan is inconsistent with the selected kernel");
    }

    void upload_plan() {
        d_slice_inst_.upload(plan_.slice_inst);
        d_inst_slice_.upload(plan_.inst_slice);
        d_cta_slice_.upload(plan_.cta_slice);
        d_cta_inst_lo_.upload(plan_.cta_inst_lo);
        d_cta_inst_hi_.upload(plan_.cta_inst_hi);
        d_inst_cta_lo_.upload(plan_.inst_cta_lo);
        d_inst_slot_.upload(plan_.inst_slot);
        d_slots_.resize((size_t)2 * std::max(1, plan_.inst_slot.back()) * kSlotW);  // two sets by phase parity
        d_fslots_.resize((size_t)3 * std::max(1, plan_.inst_slot.back()) * kSlotW);
        d_inst_.resize(plan_.n_inst);
        d_inst_.zero();
        d_bar_.resize(1);
        d_bar_.zero();
    }

    // Sizes the contact operator's buffers for the current rows.
    void prepare_contact_buffers() {
        if (!co_active_) return;
        co_rows_ = topo_.n;
        const int nb = std::max(1, grid_for(co_rows_, kScanChunk));
        d_co_cnt_.resize((size_t)co_rows_ + 1 + 4);
        d_co_cnt_.zero();
        d_co_off_.resize((size_t)co_rows_ + 1);
        d_co_bsum_.resize((size_t)nb + 1);
        d_co_ent_.resize((size_t)std::max(1, 4 * co_.max_contacts));
        d_co_rec_.resize((size_t)std::max(1, co_.max_contacts));
    }

    // The per-step contact-list build, ahead of the assembly: zero the
    // counts, prepare + count, scan, fill.  Returns the last node (or dep).
    cudaGraphNode_t add_contact_nodes(cudaGraphNode_t dep) {
        if (!co_active_) return dep;
        int dev = 0, sms = 0;
        ck(cudaGetDevice(&dev), "cudaGetDevice");
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
        const int n = co_rows_;
        const int nb = std::max(1, grid_for(n, kScanChunk));
        int* cnt = d_co_cnt_.get();
        int* stats = cnt + n + 1;
        int* off = d_co_off_.get();
        int* bsum = d_co_bsum_.get();
        int* ent = d_co_ent_.get();
        PrepContact* rec = d_co_rec_.get();
        cudaGraphNode_t last = dep;
        auto add = [&](void* fn, dim3 grid, dim3 block, void** args, const char* what) {
            cudaKernelNodeParams p{};
            p.func = fn;
            p.gridDim = grid;
            p.blockDim = block;
            p.kernelParams = args;
            cudaGraphNode_t node;
            ck(cudaGraphAddKernelNode(&node, graph_, last ? &last : nullptr, last ? 1 : 0, &p), what);
            last = node;
        };
        {
            cudaMemsetParams mp{};
            mp.dst = cnt;
            mp.value = 0;
            mp.elementSize = 4;
            mp.width = (size_t)n + 1 + 4;
            mp.height = 1;
            cudaGraphNode_t node;
            ck(cudaGraphAddMemsetNode(&node, graph_, last ? &last : nullptr, last ? 1 : 0, &mp),
               "add contact memset node");
            last = node;
        }
        ContactInput in;
        in.pairs = reinterpret_cast<const int4*>(co_.pairs);
        in.weights = reinterpret_cast<const float4*>(co_.weights);
        in.count = reinterpret_cast<const int*>(co_.count);
        in.stiffnesses = reinterpret_cast<const float*>(co_.stiffnesses);
        in.slips = reinterpret_cast<const float4*>(co_.slips);
        in.max_contacts = co_.max_contacts;
        in.stiffness = co_.stiffness;
        in.mu = co_.friction_mu;
        in.eps = co_.friction_epsilon;
        in.ext_to_row = d_ext_to_row_.get();
        int n_part = topo_.n_ext;
        const dim3 cgrid(std::max(1, std::min(grid_for(co_.max_contacts, 256), 8 * sms)));
        {
            void* a[] = {&in, &n_part, &cnt, &rec, &stats};
            add(reinterpret_cast<void*>(&contact_prep_kernel), cgrid, dim3(256), a, "add contact prep node");
        }
        int nn = n, nbb = nb;
        {
            void* a[] = {&cnt, &nn, &off, &bsum};
            add(reinterpret_cast<void*>(&contact_scan_local_kernel), dim3(nb), dim3(1024), a, "add scan node");
        }
        {
            void* a[] = {&bsum, &nbb};
            add(reinterpret_cast<void*>(&contact_scan_top_kernel), dim3(1), dim3(1024), a, "add scan node");
        }
        {
            void* a[] = {&off, &nn, &bsum, &nbb, &stats};
            add(reinterpret_cast<void*>(&contact_scan_add_kernel), dim3(std::max(1, grid_for(n, 256))), dim3(256), a,
                "add scan node");
        }
        {
            const PrepContact* crec = rec;
            const int* cstats = stats;
            const int* coff = off;
            void* a[] = {&crec, &cstats, &coff, &cnt, &ent};
            add(reinterpret_cast<void*>(&contact_fill_kernel), cgrid, dim3(256), a, "add contact fill node");
        }
        return last;
    }

    // Optional true-residual pass after the solve (off by default, as the
    // reference's compute_true_residual): a branch beside the finalize node,
    // reading b and the final x only.
    void add_true_residual_node(cudaGraphNode_t dep, DevTopo& t, Vecs& v) {
        if (!true_res_) return;
        d_tres_.resize((size_t)std::max(1, topo_.n_slices));
        double2* out = d_tres_.get();
        void* a[] = {&t, &v, &out};
        cudaKernelNodeParams p{};
        p.func = reinterpret_cast<void*>(&true_residual_kernel);
        p.gridDim = dim3(std::max(1, grid_for(std::max(1, topo_.n_slices) * 32, 256)));
        p.blockDim = dim3(256);
        p.kernelParams = a;
        cudaGraphNode_t node;
        ck(cudaGraphAddKernelNode(&node, graph_, &dep, 1, &p), "add true-residual node");
    }

    void build_graph_persistent() {
        destroy_graph();
        ck(cudaFuncSetAttribute(assemble_fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)asm_smem_),
           "cudaFuncSetAttribute(assemble smem)");
        plan_persistent();
        check_plan();
        prepare_contact_buffers();
        ck(cudaGraphCreate(&graph_, 0), "cudaGraphCreate");
        DevTopo t = dev_topo();
        ElemData el = elem_data();
        Vecs v = vecs();
        SolveState* st = d_state_.get();
        double* part = d_part_.get();
        BatchPlan bp = batch_plan();
        const bool warm = warm_mode_ != CHYSX_WARM_ZERO;
        int zero_guess = warm ? 0 : 1;
        int warm_i = warm_kernel_mode();
        cur_args_ = step_args(1.0f / 60.0f);
        cur_cfg_ = solver_cfg();
        cudaGraphConditionalHandle no_cond = 0;
        void* aargs[] = {&cur_args_, &el, &t, &v, &st, &part, &cur_cfg_, &zero_guess, &no_cond};
        cudaKernelNodeParams ap;
        asm_params(ap, aargs);
        cudaGraphNode_t t0 = add_contact_nodes(timing_node(0, nullptr));
        ck(cudaGraphAddKernelNode(&asm_node_, graph_, t0 ? &t0 : nullptr, t0 ? 1 : 0, &ap), "add assemble node");
        cudaGraphNode_t t1 = add_guess_node(asm_node_, cur_args_, t, v);
        if (coarse_on_) {
            // the coarse space and system of this step's matrix, before the solve
            CoarseArgs cg = coarse_args();
            StepArgs sa = cur_args_;
            cudaGraphNode_t prev = t1;
            cfield_node_ = nullptr;
            if (coarse_nq_ > 1) {
                void* a0[] = {&sa, &cg};
                cudaKernelNodeParams p0{};
                p0.func = reinterpret_cast<void*>(&coarse_fields_kernel);
                p0.gridDim = dim3(coarse_nb_);
                p0.blockDim = dim3(256);
                p0.kernelParams = a0;
                ck(cudaGraphAddKernelNode(&cfield_node_, graph_, &prev, 1, &p0), "add coarse fields node");
                prev = cfield_node_;
            }
            void* a1[] = {&t, &cg};
            cudaKernelNodeParams p{};
            p.func = reinterpret_cast<void*>(&coarse_assemble_kernel);
            p.gridDim = dim3(coarse_nb_, coarse_nq_, coarse_splits_);
            p.blockDim = dim3(288);
            p.sharedMemBytes = (unsigned)coarse_assemble_smem();
            p.kernelParams = a1;
            cudaGraphNode_t n1, n2;
            ck(cudaGraphAddKernelNode(&n1, graph_, &prev, 1, &p), "add coarse assemble node");
            {
                // zero the inversion's barrier and failure flag, then invert
                cudaGraphNode_t z1, z2;
                cudaMemsetParams mp{};
                mp.dst = d_cbar_.get();
                mp.value = 0;
                mp.elementSize = 4;
                mp.width = sizeof(GridBarrier) / 4;
                mp.height = 1;
                ck(cudaGraphAddMemsetNode(&z1, graph_, &n1, 1, &mp), "add coarse barrier reset node");
                mp.dst = d_cfail_.get();
                mp.width = 1;
                ck(cudaGraphAddMemsetNode(&z2, graph_, &z1, 1, &mp), "add coarse fail reset node");
                if (coarse_batched_) {
                    // one CTA per instance: the dense inverse of its coarse blocks
                    void* ab[] = {&cg};
                    cudaKernelNodeParams pb{};
                    pb.func = reinterpret_cast<void*>(&coarse_invert_batched_kernel);
                    pb.gridDim = dim3(plan_.n_inst);
                    pb.blockDim = dim3(kBatchInvThreads);
                    pb.sharedMemBytes = (unsigned)batched_invert_smem(batched_mmax_);
                    pb.kernelParams = ab;
                    ck(cudaGraphAddKernelNode(&n2, graph_, &z2, 1, &pb), "add batched coarse invert node");
                } else {
                    int dev = 0, sms = 0;
                    ck(cudaGetDevice(&dev), "cudaGetDevice");
                    ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
                    GridBarrier* gb = d_cbar_.get();
                    void* a2[] = {&cg, &gb};
                    cudaKernelNodeParams p2{};
                    // two CTAs per SM where they fit (the tile phases are latency-bound)
                    int inv_per_sm = 0;
                    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&inv_per_sm, coarse_invert_kernel,
                                                                     kCoarseInvertThreads, 0),
                       "cudaOccupancyMaxActiveBlocksPerMultiprocessor(coarse invert)");
                    p2.func = reinterpret_cast<void*>(&coarse_invert_kernel);
                    p2.gridDim = dim3(sms * std::max(1, std::min(2, inv_per_sm)));
                    p2.blockDim = dim3(kCoarseInvertThreads);
                    p2.kernelParams = a2;
                    ck(cudaGraphAddKernelNode(&n2, graph_, &z2, 1, &p2), "add coarse invert node");
                    cudaLaunchAttributeValue coop{};
                    coop.cooperative = 1;
                    ck(cudaGraphKernelNodeSetAttribute(n2, cudaLaunchAttributeCooperative, &coop),
                       "cooperative attribute (coarse invert)");
                }
            }
            t1 = n2;
        }
        t1 = timing_node(1, t1);
        cudaGraphNode_t reset;
        {
            void* rargs[] = {&bp};
            cudaKernelNodeParams p{};
            p.func = reinterpret_cast<void*>(&pcg_persistent_reset_kernel);
            p.gridDim = dim3(grid_for(std::max(std::max(1, plan_.n_inst), 3 * kSlotW * bp.n_slots), 256));
            p.blockDim = dim3(256);
            p.kernelParams = rargs;
            ck(cudaGraphAddKernelNode(&reset, graph_, &t1, 1, &p), "add reset node");
        }
        {
            void* ex0 = exchange_buffer(0);
            void* ex1 = exchange_buffer(1);
            void* pargs[] = {&t, &v, &bp, &cur_cfg_, &warm_i, &ex0, &ex1};
            cudaKernelNodeParams p{};
            p.func = const_cast<void*>(persistent_fn());
            p.gridDim = dim3(plan_.grid);
            p.blockDim = dim3(resident_ ? resident_warps_ * 32 : pcg_block_);
            p.sharedMemBytes = (unsigned)pers_smem_;
            p.kernelParams = pargs;
            ck(cudaGraphAddKernelNode(&pcg_node_, graph_, &reset, 1, &p), "add persistent PCG node");
            cudaLaunchAttributeValue coop{};
            coop.cooperative = 1;
            ck(cudaGraphKernelNodeSetAttribute(pcg_node_, cudaLaunchAttributeCooperative, &coop),
               "cooperative attribute");
        }
        {
            const int vgrid = std::max(1, grid_for(topo_.n, kVecBlock));
            void* fargs[] = {&cur_args_, &v, &bp};
            cudaKernelNodeParams p{};
            p.func = reinterpret_cast<void*>(&finalize_batch_kernel);
            p.gridDim = dim3(vgrid);
            p.blockDim = dim3(kVecBlock);
            p.kernelParams = fargs;
            cudaGraphNode_t t2 = timing_node(2, pcg_node_);
            ck(cudaGraphAddKernelNode(&fin_node_, graph_, &t2, 1, &p), "add finalize node");
            timing_node(3, fin_node_);
        }
        add_true_residual_node(pcg_node_, t, v);
        ck(cudaGraphInstantiate(&exec_, graph_, 0), "cudaGraphInstantiate(step)");
        graph_path_ = kPathPersistent;
        graph_dirty_ = false;
        node_args_ = cur_args_;
        node_cfg_ = cur_cfg_;
        nodes_valid_ = true;
    }

    void build_graph_loop() {
        destroy_graph();
        ck(cudaFuncSetAttribute(assemble_fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)asm_smem_),
           "cudaFuncSetAttribute(assemble smem)");
        prepare_contact_buffers();
        ck(cudaGraphCreate(&graph_, 0), "cudaGraphCreate");
        ck(cudaGraphConditionalHandleCreate(&cond_, graph_, 1, cudaGraphCondAssignDefault),
           "cudaGraphConditionalHandleCreate");
        DevTopo t = dev_topo();
        ElemData el = elem_data();
        Vecs v = vecs();
        SolveState* st = d_state_.get();
        double* part = d_part_.get();
        const bool warm = warm_mode_ != CHYSX_WARM_ZERO;
        int zero_guess = warm ? 0 : 1;
        cur_args_ = step_args(1.0f / 60.0f);
        cur_cfg_ = solver_cfg();
        cudaGraphConditionalHandle cond = cond_;

        void* aargs[] = {&cur_args_, &el, &t, &v, &st, &part, &cur_cfg_, &zero_guess, &cond};
        cudaKernelNodeParams ap;
        asm_params(ap, aargs);
        cudaGraphNode_t t0 = add_contact_nodes(timing_node(0, nullptr));
        ck(cudaGraphAddKernelNode(&asm_node_, graph_, t0 ? &t0 : nullptr, t0 ? 1 : 0, &ap), "add assemble node");
        cudaGraphNode_t last = add_guess_node(asm_node_, cur_args_, t, v);
        last = timing_node(1, last);

        const int vgrid = std::max(1, grid_for(topo_.n, kVecBlock));
        if (warm) {
            cudaKernelNodeParams p{};
            int scaled = warm_kernel_mode() == 2 ? 1 : 0;
            void* iargs[] = {&t, &v, &st, &part, &cond, &scaled};
            p.func = reinterpret_cast<void*>(&warm_init_kernel<kVecBlock>);
            p.gridDim = dim3(vgrid);
            p.blockDim = dim3(kVecBlock);
            p.kernelParams = iargs;
            cudaGraphNode_t n1;
            ck(cudaGraphAddKernelNode(&n1, graph_, &last, 1, &p), "add warm_init node");
            void* fargs[] = {&t, &v, &st};
            cudaKernelNodeParams pf{};
            pf.func = reinterpret_cast<void*>(&warm_fixup_kernel);
            pf.gridDim = dim3(vgrid);
            pf.blockDim = dim3(kVecBlock);
            pf.kernelParams = fargs;
            cudaGraphNode_t n2;
            ck(cudaGraphAddKernelNode(&n2, graph_, &n1, 1, &pf), "add warm_fixup node");
            last = n2;
        }
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond_;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t loop;
        ck(cudaGraphAddNode(&loop, graph_, &last, 1, &cp), "add while node");
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        {
            void* kargs[] = {&t, &v, &st, &part, &cond};
            cudaKernelNodeParams p1{};
            p1.func = reinterpret_cast<void*>(&pcg_spmv_kernel<kVecBlock>);
            p1.gridDim = dim3(vgrid);
            p1.blockDim = dim3(kVecBlock);
            p1.kernelParams = kargs;
            cudaGraphNode_t k1;
            ck(cudaGraphAddKernelNode(&k1, body, nullptr, 0, &p1), "add pcg_spmv node");
            cudaKernelNodeParams p2 = p1;
            p2.func = reinterpret_cast<void*>(&pcg_update_kernel<kVecBlock>);
            cudaGraphNode_t k2;
            ck(cudaGraphAddKernelNode(&k2, body, &k1, 1, &p2), "add pcg_update node");
        }
        {
            void* fargs[] = {&cur_args_, &v, &st};
            cudaKernelNodeParams p{};
            p.func = reinterpret_cast<void*>(&finalize_kernel);
            p.gridDim = dim3(vgrid);
            p.blockDim = dim3(kVecBlock);
            p.kernelParams = fargs;
            cudaGraphNode_t t2 = timing_node(2, loop);
            ck(cudaGraphAddKernelNode(&fin_node_, graph_, &t2, 1, &p), "add finalize node");
            timing_node(3, fin_node_);
        }
        add_true_residual_node(loop, t, v);
        ck(cudaGraphInstantiate(&exec_, graph_, 0), "cudaGraphInstantiate(step)");
        graph_path_ = kPathLoop;
        graph_dirty_ = false;
        // node args as instantiated; the first step patches them
        node_args_ = cur_args_;
        node_cfg_ = cur_cfg_;
        nodes_valid_ = true;
    }

    void update_step_nodes(float dt) {
        StepArgs a = step_args(dt);
        SolverCfg c = solver_cfg();
        if (nodes_valid_ && same_bytes(a, node_args_) && same_bytes(c, node_cfg_)) return;
        DevTopo t = dev_topo();
        ElemData el = elem_data();
        Vecs v = vecs();
        SolveState* st = d_state_.get();
        double* part = d_part_.get();
        int zero_guess = warm_mode_ != CHYSX_WARM_ZERO ? 0 : 1;
        if (graph_path_ == kPathPersistent) {
            cudaGraphConditionalHandle no_cond = 0;
            BatchPlan bp = batch_plan();
            int warm_i = warm_kernel_mode();
            void* aargs[] = {&a, &el, &t, &v, &st, &part, &c, &zero_guess, &no_cond};
            cudaKernelNodeParams ap;
            asm_params(ap, aargs);
            ck(cudaGraphExecKernelNodeSetParams(exec_, asm_node_, &ap), "update assemble node");
            void* ex0 = exchange_buffer(0);
            void* ex1 = exchange_buffer(1);
            void* pargs[] = {&t, &v, &bp, &c, &warm_i, &ex0, &ex1};
            cudaKernelNodeParams pp{};
            pp.func = const_cast<void*>(persistent_fn());
            pp.gridDim = dim3(plan_.grid);
            pp.blockDim = dim3(resident_ ? resident_warps_ * 32 : pcg_block_);
            pp.sharedMemBytes = (unsigned)pers_smem_;
            pp.kernelParams = pargs;
            ck(cudaGraphExecKernelNodeSetParams(exec_, pcg_node_, &pp), "update persistent PCG node");
            void* fargs[] = {&a, &v, &bp};
            cudaKernelNodeParams fp{};
            fp.func = reinterpret_cast<void*>(&finalize_batch_kernel);
            fp.gridDim = dim3(std::max(1, grid_for(topo_.n, kVecBlock)));
            fp.blockDim = dim3(kVecBlock);
            fp.kernelParams = fargs;
            ck(cudaGraphExecKernelNodeSetParams(exec_, fin_node_, &fp), "update finalize node");
            if (coarse_on_ && cfield_node_) {  // the coarse fields read x_n
                CoarseArgs cg = coarse_args();
                void* cargs[] = {&a, &cg};
                cudaKernelNodeParams cp{};
                cp.func = reinterpret_cast<void*>(&coarse_fields_kernel);
                cp.gridDim = dim3(coarse_nb_);
                cp.blockDim = dim3(256);
                cp.kernelParams = cargs;
                ck(cudaGraphExecKernelNodeSetParams(exec_, cfield_node_, &cp), "update coarse fields node");
            }
            patch_guess_node(a, t, v);
            node_args_ = a;
            node_cfg_ = c;
            nodes_valid_ = true;
            return;
        }
        cudaGraphConditionalHandle cond = cond_;
        void* aargs[] = {&a, &el, &t, &v, &st, &part, &c, &zero_guess, &cond};
        cudaKernelNodeParams ap;
        asm_params(ap, aargs);
        ck(cudaGraphExecKernelNodeSetParams(exec_, asm_node_, &ap), "update assemble node");
        const int vgrid = std::max(1, grid_for(topo_.n, kVecBlock));
        void* fargs[] = {&a, &v, &st};
        cudaKernelNodeParams p{};
        p.func = reinterpret_cast<void*>(&finalize_kernel);
        p.gridDim = dim3(vgrid);
        p.blockDim = dim3(kVecBlock);
        p.kernelParams = fargs;
        ck(cudaGraphExecKernelNodeSetParams(exec_, fin_node_, &p), "update finalize node");
        patch_guess_node(a, t, v);
        node_args_ = a;
        node_cfg_ = c;
        nodes_valid_ = true;
    }

    // caller buffers
    uintptr_t pos_ = 0, vel_ = 0, inv_mass_ = 0, force_ = 0;
    uintptr_t pos_out_ = 0, vel_out_ = 0;  // step_into's outputs, for that call only
    int n_ = 0;
    // mesh
    std::vector<int> tris_, edges_;
    DevBuf<int> d_tris_, d_edges_, d_vt_off_, d_vt_list_;
    int vt_n_ = -1;
    bool mesh_on_device_ = false;
    // elements
    bool springs_built_ = false, stretch_built_ = false, shear_built_ = false;
    DevBuf<double> d_rest_;
    DevBuf<float> d_kedge_, d_area_, d_ktri_, d_area_s_, d_ktri_s_;
    DevBuf<RestShape> d_dminv_, d_dminv_s_;
    std::vector<int> pin_idx_;
    std::vector<float> pin_tgt_;
    float pin_k_ = 1.0e6f;
    // options (defaults reproduce the reference)
    bool springs_in_step_ = true, apply_force_ = false;
    float det_eps_ = 1.0e-6f;
    int max_iter_ = 50;
    double rel_tol_ = 0.0;
    int warm_mode_ = CHYSX_WARM_PREVIOUS;
    // topology + system
    bool topo_dirty_ = true, use_tris_ = false, use_stretch_ = false, use_shear_ = false, use_springs_ = false;
    bool bending_built_ = false, use_bending_ = false;
    float k_bend_ = 0.0f;
    std::vector<int> dih_;
    DevBuf<int4> d_dih_;
    DevBuf<double> d_rest_angle_;
    DevBuf<int> d_dinc_off_, d_dinc_;
    DevBuf<unsigned> d_dinc_meta_;
    // floats per stored off-diagonal block: bending makes them unsymmetric
    int off_width() const { return use_bending_ ? 9 : 6; }
    HostTopology topo_;
    DevBuf<int> d_slice_off_, d_col_, d_tinc_off_, d_tinc_, d_sinc_off_, d_sinc_, d_pin_off_, d_pin_row_;
    DevBuf<unsigned> d_tinc_meta_, d_sinc_meta_;
    DevBuf<float> d_val_, d_diag_, d_dnl_, d_minv_, d_pin_tgt_;
    DevBuf<float4> d_b_, d_r_, d_z_, d_x_, d_ap_, d_p0_, d_p1_;
    DevBuf<double> d_part_;
    DevBuf<SolveState> d_state_;
    int asm_block_ = 128;
    size_t asm_smem_ = 0;
    static constexpr size_t kMaxAssembleSmem = 227 * 1024;  // dynamic shared memory of one CTA
    // persistent PCG plan
    static constexpr int kPathPersistent = 0, kPathLoop = 1, kPathStreamed = 2;
    int solver_path_ = kPathPersistent, graph_path_ = kPathPersistent;
    int pcg_block_ = 256, pcg_grid_req_ = 0;
    int pcg_block_req_ = 0;  // the caller's block size (0: chosen by the planner)
    HostPlan plan_;
    size_t pers_smem_ = 0;
    DevBuf<int> d_slice_inst_, d_inst_slice_, d_cta_slice_, d_cta_inst_lo_, d_cta_inst_hi_, d_inst_cta_lo_,
        d_inst_slot_;
    DevBuf<double> d_slots_;
    DevBuf<unsigned long long> d_fslots_;
    DevBuf<InstState> d_inst_;
    DevBuf<GridBarrier> d_bar_;
    cudaGraphNode_t pcg_node_ = nullptr;
    DevBuf<float> d_net_params_;
    DevBuf<MlpPacked> d_net_;
    uintptr_t feat_out_ = 0, pred_out_ = 0;
    cudaGraphNode_t guess_node_ = nullptr;
    std::vector<int> inst_offsets_;
    DevBuf<int> d_row_to_ext_, d_ext_to_row_;
    int row_order_ = 0;
    std::vector<int> order_;  // particles in row order (row_order_ 1)
    bool resident_ = false;
    int resident_warps_ = 16;
    std::vector<TuneResult> tune_;
    int sync_mode_ = 0;    // 0 grid counter barrier, 1 polled per-instance slots
    int pc_kind_ = 0, pc_degree_ = 0;  // preconditioner: 0 block-Jacobi, 1 CTA-local Chebyshev, 2 + coarse level
    bool coarse_on_ = false;
    int coarse_nb_ = 0, coarse_mn_ = 0, coarse_g_ = 1, coarse_nq_ = 1, coarse_splits_ = 1;
    bool coarse_batched_ = false;  // the streamed kernel's per-instance level (plan_coarse_batched)
    int batched_mmax_ = 0;         // its largest per-instance inverse
    DevBuf<int> d_blk_slot_, d_inst_blk_, d_inst_aoff_, d_slot_cb_;
    double coarse_shift_ = 0.0;
    DevBuf<int> d_slice_cb_, d_cb_row0_, d_cnbr_, d_ccnt_, d_cself_;
    DevBuf<unsigned char> d_ell_nbr_;
    DevBuf<float4> d_cw_;
    DevBuf<CoarseArgs> d_cargs_;  // the coarse arguments the PCG kernel reads (BatchPlan holds the pointer)
    DevBuf<float> d_cac_, d_cainv_;
    DevBuf<double> d_cacp_;  // the coarse assembly's per-split partial sums
    DevBuf<double> d_cwork_;
    DevBuf<int> d_cfail_;
    DevBuf<GridBarrier> d_cbar_;
    float pc_ratio_ = 0.0f;
    DevBuf<ZP> d_zp_;
    bool timing_ = false;
    cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
    bool true_res_ = false;
    DevBuf<double2> d_tres_;  // per-slice (r.r, b.b) of the true-residual pass
    // static shapes: planes (n, d), boxes (center, half extents, axes)
    std::vector<float> planes_, boxes_;
    float sc_thickness_ = 0.0f, sc_k_ = 0.0f, sc_mu_ = 0.0f, sc_eps_ = 1.0e-4f;
    bool static_dirty_ = false;
    DevBuf<float> d_shapes_;
    // contact operator and its per-step row lists
    chysx_contact_op co_{};
    bool co_active_ = false;
    int co_rows_ = 0;           // rows of the lists at the last graph build
    DevBuf<int> d_co_cnt_;      // [rows + 1] counts, then 4 stats ints
    DevBuf<int> d_co_off_, d_co_bsum_, d_co_ent_;
    DevBuf<PrepContact> d_co_rec_;
    // graph
    bool graph_dirty_ = true, nodes_valid_ = false;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    cudaGraphNode_t asm_node_ = nullptr, fin_node_ = nullptr;
    cudaGraphNode_t cfield_node_ = nullptr;  // coarse fields (two-level preconditioner with linear fields)
    cudaGraphConditionalHandle cond_ = 0;
    StepArgs cur_args_{}, node_args_{};
    SolverCfg cur_cfg_{}, node_cfg_{};
    uintptr_t last_stream_ = 0;
    bool stepped_ = false;
};

}  // namespace chysx_b200

#include "vbd_host.cuh"

// ===========================================================================
// C ABI
// ===========================================================================
using chysx_b200::ClothSim;
using chysx_b200::VbdSolver;

struct chysx_vbd {
    VbdSolver solver;
};

struct chysx_cloth {
    ClothSim sim;
};

namespace {

template <class F>
int guard(F&& f) {
    try {
        f();
        return CHYSX_OK;
    } catch (const std::invalid_argument& e) {
        chysx_b200::g_err = e.what();
        return CHYSX_ERR_INVALID_ARGUMENT;
    } catch (const std::out_of_range& e) {
        chysx_b200::g_err = e.what();
        return CHYSX_ERR_OUT_OF_RANGE;
    } catch (const chysx_b200::CudaFailure& e) {
        chysx_b200::g_err = e.what();
        return CHYSX_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        chysx_b200::g_err = "host allocation failed";
        return CHYSX_ERR_RUNTIME;
    } catch (const std::exception& e) {
        chysx_b200::g_err = e.what();
        return CHYSX_ERR_RUNTIME;
    }
}

int null_handle() {
    chysx_b200::g_err = "null chysx_cloth handle";
    return CHYSX_ERR_INVALID_ARGUMENT;
}

}  // namespace

#define CHYSX_H(h)            \
    if (!(h)) return null_handle()

extern "C" {

const char* chysx_last_error(void) { return chysx_b200::g_err.c_str(); }

int chysx_cloth_create(chysx_cloth** out) {
    if (!out) return null_handle();
    return guard([&] { *out = new chysx_cloth(); });
}
int chysx_cloth_destroy(chysx_cloth* h) {
    delete h;
    return CHYSX_OK;
}
int chysx_cloth_set_material(chysx_cloth* h, const chysx_cloth_material* m) {
    CHYSX_H(h);
    if (!m) return null_handle();
    h->sim.mat = *m;
    return CHYSX_OK;
}
int chysx_cloth_get_material(const chysx_cloth* h, chysx_cloth_material* out) {
    CHYSX_H(h);
    if (!out) return null_handle();
    *out = h->sim.mat;
    return CHYSX_OK;
}
int chysx_cloth_set_external_buffers(chysx_cloth* h, uintptr_t pos, uintptr_t vel, int count,
                                     uintptr_t inv_mass, uintptr_t force) {
    CHYSX_H(h);
    h->sim.set_external_buffers(pos, vel, count, inv_mass, force);
    return CHYSX_OK;
}
int chysx_cloth_set_mesh(chysx_cloth* h, const int32_t* tris, int n) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_mesh(tris, n); });
}
int chysx_cloth_num_edges(const chysx_cloth* h, int* out) {
    CHYSX_H(h);
    if (out) *out = h->sim.num_edges();
    return CHYSX_OK;
}
int chysx_cloth_get_edges(const chysx_cloth* h, int32_t* out) {
    CHYSX_H(h);
    if (out) std::copy(h->sim.edges().begin(), h->sim.edges().end(), out);
    return CHYSX_OK;
}
int chysx_cloth_set_pins(chysx_cloth* h, const int32_t* idx, const float* targets, int n, float k) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_pins(idx, targets, n, k); });
}
int chysx_cloth_clear_pins(chysx_cloth* h) {
    CHYSX_H(h);
    h->sim.clear_pins();
    return CHYSX_OK;
}
int chysx_cloth_num_pins(const chysx_cloth* h, int* out) {
    CHYSX_H(h);
    if (out) *out = h->sim.num_pins();
    return CHYSX_OK;
}
int chysx_cloth_update_pin_targets(chysx_cloth* h, const float* targets, int n, uintptr_t stream) {
    CHYSX_H(h);
    return guard([&] { h->sim.update_pin_targets(targets, n, stream); });
}
int chysx_cloth_build_springs(chysx_cloth* h, float k, const float* k_per_edge, uintptr_t stream) {
    CHYSX_H(h);
    return guard([&] { h->sim.build_springs(k, k_per_edge, stream); });
}
int chysx_cloth_num_springs(const chysx_cloth* h, int* out) {
    CHYSX_H(h);
    if (out) *out = h->sim.num_springs();
    return CHYSX_OK;
}
int chysx_cloth_build_fem_stretch(chysx_cloth* h, float k, const float* k_per_tri, uintptr_t stream) {
    CHYSX_H(h);
    return guard([&] { h->sim.build_stretch(k, k_per_tri, stream); });
}
int chysx_cloth_build_fem_shear(chysx_cloth* h, float k, const float* k_per_tri, uintptr_t stream) {
    CHYSX_H(h);
    return guard([&] { h->sim.build_shear(k, k_per_tri, stream); });
}
int chysx_cloth_build_bending(chysx_cloth* h, float k, uintptr_t stream) {
    CHYSX_H(h);
    return guard([&] { h->sim.build_bending(k, stream); });
}
int chysx_cloth_num_dihedrals(const chysx_cloth* h, int* out) {
    CHYSX_H(h);
    if (out) *out = h->sim.num_dihedrals();
    return CHYSX_OK;
}
int chysx_cloth_add_static_plane(chysx_cloth* h, const float* n, float d) {
    CHYSX_H(h);
    return guard([&] { h->sim.add_static_plane(n, d); });
}
int chysx_cloth_add_static_box(chysx_cloth* h, const float* c, const float* he, const float* ex, const float* ey,
                               const float* ez) {
    CHYSX_H(h);
    return guard([&] { h->sim.add_static_box(c, he, ex, ey, ez); });
}
int chysx_cloth_clear_static_shapes(chysx_cloth* h) {
    CHYSX_H(h);
    h->sim.clear_static_shapes();
    return CHYSX_OK;
}
int chysx_cloth_static_shape_counts(const chysx_cloth* h, int* planes, int* boxes) {
    CHYSX_H(h);
    if (planes) *planes = h->sim.static_planes();
    if (boxes) *boxes = h->sim.static_boxes();
    return CHYSX_OK;
}
int chysx_cloth_set_static_contact_thickness(chysx_cloth* h, float t) {
    CHYSX_H(h);
    h->sim.set_static_param(0, t);
    return CHYSX_OK;
}
int chysx_cloth_set_static_contact_stiffness(chysx_cloth* h, float k) {
    CHYSX_H(h);
    h->sim.set_static_param(1, k);
    return CHYSX_OK;
}
int chysx_cloth_set_static_contact_friction(chysx_cloth* h, float mu) {
    CHYSX_H(h);
    h->sim.set_static_param(2, mu);
    return CHYSX_OK;
}
int chysx_cloth_set_static_contact_friction_epsilon(chysx_cloth* h, float eps) {
    CHYSX_H(h);
    h->sim.set_static_param(3, eps);
    return CHYSX_OK;
}
int chysx_cloth_get_static_contact(const chysx_cloth* h, float* t, float* k, float* mu, float* eps) {
    CHYSX_H(h);
    h->sim.get_static_params(t, k, mu, eps);
    return CHYSX_OK;
}
int chysx_cloth_set_contact_op(chysx_cloth* h, const chysx_contact_op* op) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_contact_op(op); });
}
int chysx_cloth_clear_contact_op(chysx_cloth* h) {
    CHYSX_H(h);
    h->sim.clear_contact_op();
    return CHYSX_OK;
}
int chysx_cloth_contact_stats(chysx_cloth* h, int* live, int* dropped, int* slots) {
    CHYSX_H(h);
    return guard([&] { h->sim.contact_stats(live, dropped, slots); });
}
int chysx_cloth_redistribute_mass(chysx_cloth* h, float rho, uintptr_t inv_mass, int n, uintptr_t stream) {
    CHYSX_H(h);
    return guard([&] { h->sim.redistribute_mass(rho, inv_mass, n, stream); });
}
int chysx_cloth_set_pcg_iterations(chysx_cloth* h, int m) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_pcg_iterations(m); });
}
int chysx_cloth_pcg_iterations(const chysx_cloth* h, int* out) {
    CHYSX_H(h);
    if (out) *out = h->sim.pcg_iterations();
    return CHYSX_OK;
}
int chysx_cloth_set_solver(chysx_cloth* h, int max_iter, double rel_tol, int warm) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_solver(max_iter, rel_tol, warm); });
}
int chysx_cloth_set_options(chysx_cloth* h, int sis, int af, float eps) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_options(sis, af, eps); });
}
int chysx_cloth_step(chysx_cloth* h, float dt, uintptr_t stream) {
    CHYSX_H(h);
    return guard([&] { h->sim.step(dt, stream); });
}
int chysx_cloth_step_into(chysx_cloth* h, float dt, uintptr_t pos_in, uintptr_t vel_in, uintptr_t pos_out,
                          uintptr_t vel_out, uintptr_t stream) {
    CHYSX_H(h);
    return guard([&] { h->sim.step_into(dt, pos_in, vel_in, pos_out, vel_out, stream); });
}
int chysx_cloth_last_stats(chysx_cloth* h, int* iters, double* relres, int* status) {
    CHYSX_H(h);
    return guard([&] { h->sim.last_stats(iters, relres, status); });
}
int chysx_cloth_set_true_residual(chysx_cloth* h, int on) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_true_residual(on); });
}
int chysx_cloth_true_residual(chysx_cloth* h, int n_instances, double* relres, double* worst) {
    CHYSX_H(h);
    return guard([&] { h->sim.true_residual(n_instances, relres, worst); });
}
int chysx_cloth_num_particles(const chysx_cloth* h, int* out) {
    CHYSX_H(h);
    if (out) *out = h->sim.num_particles();
    return CHYSX_OK;
}
int chysx_cloth_num_off_diag_blocks(const chysx_cloth* h, int* out) {
    CHYSX_H(h);
    if (out) *out = h->sim.num_off_diag_blocks();
    return CHYSX_OK;
}
int chysx_cloth_debug_dump(chysx_cloth* h, float* diag, int32_t* rp, int32_t* col, float* vals, float* rhs,
                           float* dx) {
    CHYSX_H(h);
    return guard([&] { h->sim.debug_dump(diag, rp, col, vals, rhs, dx); });
}

int chysx_cloth_debug_coarse(chysx_cloth* h, int32_t* info, float* ac, float* ainv, int cap) {
    CHYSX_H(h);
    return guard([&] { h->sim.debug_coarse(info, ac, ainv, cap); });
}
int chysx_cloth_debug_coarse_rows(chysx_cloth* h, int32_t* row0, int cap, int32_t* count) {
    CHYSX_H(h);
    return guard([&] {
        if (!count) throw std::invalid_argument("debug_coarse_rows: null count");
        *count = h->sim.debug_coarse_rows(row0, cap);
    });
}

int chysx_cloth_set_network(chysx_cloth* h, const float* params, int n_params) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_network(params, n_params); });
}
int chysx_cloth_set_feature_output(chysx_cloth* h, uintptr_t features, uintptr_t predictions) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_feature_output(features, predictions); });
}
int chysx_cloth_guess_kept(chysx_cloth* h, int* kept) {
    CHYSX_H(h);
    return guard([&] {
        const int k = h->sim.guess_kept();
        if (kept) *kept = k;
    });
}
int chysx_mlp_num_params(void) { return chysx_b200::MlpOffsets::total; }
int chysx_mlp_num_features(void) { return chysx_b200::kMlpIn; }
uint64_t chysx_mlp_workspace_bytes(int rows) { return chysx_b200::mlp_workspace_bytes(rows); }
int chysx_mlp_gradients(uintptr_t params, uintptr_t features, uintptr_t targets, int rows, uintptr_t grad,
                        double* loss, uintptr_t workspace, uint64_t workspace_bytes, uintptr_t stream) {
    return guard([&] {
        chysx_b200::mlp_gradients(params, features, targets, rows, grad, loss, 0, workspace, workspace_bytes,
                                  stream);
    });
}
int chysx_mlp_predict(uintptr_t params, uintptr_t features, int rows, uintptr_t dv, uintptr_t workspace,
                      uint64_t workspace_bytes, uintptr_t stream) {
    return guard([&] {
        chysx_b200::mlp_gradients(params, features, 0, rows, 0, nullptr, dv, workspace, workspace_bytes, stream);
    });
}
int chysx_mlp_train_step(uintptr_t params, uintptr_t grad, uintptr_t m1, uintptr_t m2, uintptr_t features,
                         uintptr_t targets, int rows, float lr, int adam_step, uintptr_t workspace,
                         uint64_t workspace_bytes, double* loss, uintptr_t stream) {
    return guard([&] {
        chysx_b200::mlp_gradients(params, features, targets, rows, grad, loss, 0, workspace, workspace_bytes,
                                  stream);
        chysx_b200::mlp_adam(params, grad, m1, m2, lr, adam_step, stream);
    });
}
int chysx_mlp_noalloc_max_rows(void) { return CHYSX_MLP_NOALLOC_MAX_ROWS; }
int chysx_mlp_gradients_noalloc(uintptr_t params, uintptr_t features, uintptr_t targets, int rows,
                                uintptr_t grad, double* loss, uintptr_t stream) {
    return guard([&] { chysx_b200::mlp_gradients_noalloc(params, features, targets, rows, grad, loss, stream); });
}
int chysx_cloth_set_instances(chysx_cloth* h, const int32_t* offsets, int n_instances) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_instances(offsets, n_instances); });
}
int chysx_cloth_num_instances(const chysx_cloth* h, int* out) {
    CHYSX_H(h);
    if (out) *out = h->sim.num_instances();
    return CHYSX_OK;
}
int chysx_cloth_instance_stats(chysx_cloth* h, int n, int* iters, double* relres, int* status) {
    CHYSX_H(h);
    return guard([&] { h->sim.instance_stats(n, iters, relres, status); });
}
int chysx_cloth_autotune(chysx_cloth* h, float dt, int repetitions, uintptr_t stream) {
    CHYSX_H(h);
    return guard([&] { h->sim.autotune(dt, repetitions, stream); });
}
int chysx_cloth_autotune_results(const chysx_cloth* h, int capacity, int* count, int32_t* config,
                                 float* solve_ms) {
    CHYSX_H(h);
    const auto& t = h->sim.tune_results();
    if (count) *count = (int)t.size();
    for (int k = 0; k < std::min(capacity, (int)t.size()); ++k) {
        if (config) {
            int32_t* c = config + 8 * (size_t)k;
            c[0] = t[k].path; c[1] = t[k].block; c[2] = t[k].sync;
            c[3] = t[k].used; c[4] = t[k].used_grid; c[5] = t[k].used_block; c[6] = t[k].iters; c[7] = t[k].status;
        }
        if (solve_ms) solve_ms[k] = t[k].solve_ms;
    }
    return CHYSX_OK;
}
int chysx_cloth_set_sync_mode(chysx_cloth* h, int mode) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_sync(mode); });
}
int chysx_cloth_sync_mode(const chysx_cloth* h, int* mode) {
    CHYSX_H(h);
    if (mode) *mode = h->sim.sync_mode();
    return CHYSX_OK;
}
int chysx_cloth_set_tuning(chysx_cloth* h, int solver_path, int block, int grid) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_tuning(solver_path, block, grid); });
}
int chysx_cloth_set_row_order(chysx_cloth* h, int mode) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_row_order(mode); });
}
int chysx_cloth_row_of_particles(const chysx_cloth* h, int n, int32_t* rows) {
    CHYSX_H(h);
    return guard([&] { h->sim.row_of_particles(n, rows); });
}
int chysx_cloth_set_preconditioner(chysx_cloth* h, int kind, int degree, float ratio) {
    CHYSX_H(h);
    return guard([&] { h->sim.set_preconditioner(kind, degree, ratio); });
}
int chysx_cloth_preconditioner(const chysx_cloth* h, int* kind, int* degree, float* ratio, int* in_use) {
    CHYSX_H(h);
    h->sim.preconditioner(kind, degree, ratio, in_use);
    return CHYSX_OK;
}
int chysx_cloth_solver_info(const chysx_cloth* h, int* path, int* grid, int* block) {
    CHYSX_H(h);
    h->sim.solver_info(path, grid, block);
    return CHYSX_OK;
}

int chysx_cloth_enable_timing(chysx_cloth* h, int on) {
    CHYSX_H(h);
    return guard([&] { h->sim.enable_timing(on); });
}
int chysx_cloth_last_timing(chysx_cloth* h, float* assemble_ms, float* solve_ms, float* finalize_ms) {
    CHYSX_H(h);
    return guard([&] { h->sim.last_timing(assemble_ms, solve_ms, finalize_ms); });
}

int chysx_topology_pattern(int n, const int32_t* tris, int n_tris, const int32_t* edges, int n_edges,
                           int32_t* row_offsets, int32_t* col_indices, int max_nnz, int* nnz_out,
                           int* ell_entries_out, int* max_width_out) {
    return guard([&] {
        std::vector<int> t(tris, tris + 3 * (size_t)std::max(0, n_tris));
        std::vector<int> e(edges, edges + 2 * (size_t)std::max(0, n_edges));
        chysx_b200::HostTopology topo;
        chysx_b200::build_topology(n, t, n_tris > 0, e, n_edges > 0, {}, {}, topo);
        if (nnz_out) *nnz_out = (int)topo.nnz();
        if (ell_entries_out) *ell_entries_out = (int)topo.ell_entries();
        if (max_width_out) *max_width_out = topo.max_width;
        if (row_offsets) std::copy(topo.csr_ptr.begin(), topo.csr_ptr.end(), row_offsets);
        if (col_indices) {
            if (topo.nnz() > max_nnz) throw std::invalid_argument("chysx_topology_pattern: col_indices too small");
            std::copy(topo.csr_col.begin(), topo.csr_col.end(), col_indices);
        }
    });
}

// ---- cloth VBD solver (include/chysx_vbd.h) -------------------------------
#define CHYSX_VBD(h)          \
    if (!(h)) return null_handle()

int chysx_vbd_create(chysx_vbd** out) {
    if (!out) return null_handle();
    return guard([&] { *out = new chysx_vbd(); });
}
int chysx_vbd_destroy(chysx_vbd* h) {
    delete h;
    return CHYSX_OK;
}
int chysx_vbd_build_cloth_coloring(chysx_vbd* h, const int32_t* tris, int n_tris, const int32_t* edges, int n_edges,
                                   int n_particles) {
    CHYSX_VBD(h);
    return guard([&] { h->solver.build_cloth_coloring(tris, n_tris, edges, n_edges, n_particles); });
}
int chysx_vbd_set_coloring(chysx_vbd* h, const int32_t* colors, int n_particles) {
    CHYSX_VBD(h);
    return guard([&] { h->solver.set_coloring(colors, n_particles); });
}
int chysx_vbd_build_tri_adjacency(chysx_vbd* h, const int32_t* tris, int n_tris, int n_particles) {
    CHYSX_VBD(h);
    return guard([&] { h->solver.build_tri_adjacency(tris, n_tris, n_particles); });
}
int chysx_vbd_build_edge_adjacency(chysx_vbd* h, const int32_t* edges, int n_edges, int n_particles) {
    CHYSX_VBD(h);
    return guard([&] { h->solver.build_edge_adjacency(edges, n_edges, n_particles); });
}
int chysx_vbd_num_colors(const chysx_vbd* h, int* out) {
    CHYSX_VBD(h);
    if (out) *out = h->solver.num_colors();
    return CHYSX_OK;
}
int chysx_vbd_colors(const chysx_vbd* h, int32_t* out, int n_particles) {
    CHYSX_VBD(h);
    return guard([&] { h->solver.colors(out, n_particles); });
}
int chysx_vbd_step_cloth(chysx_vbd* h, uintptr_t pos, uintptr_t vel, uintptr_t inv_mass, int n_particles,
                         uintptr_t tri_indices, uintptr_t tri_poses, uintptr_t tri_areas, uintptr_t tri_materials,
                         int n_tris, uintptr_t edge_indices, uintptr_t edge_rest_angle, uintptr_t edge_rest_length,
                         uintptr_t edge_bending_props, int n_edges, float gx, float gy, float gz, float dt,
                         int iterations, uintptr_t stream) {
    CHYSX_VBD(h);
    return guard([&] {
        h->solver.step_cloth(pos, vel, inv_mass, n_particles, tri_indices, tri_poses, tri_areas, tri_materials, n_tris,
                             edge_indices, edge_rest_angle, edge_rest_length, edge_bending_props, n_edges, gx, gy, gz,
                             dt, iterations, stream);
    });
}

}  // extern "C"
