// bec_api.cpp -- host side of the engine: the C ABI of include/bec.h.
//
// Replaces the reference's host driver (programs/bec_wigner_3d.cuda/wigner.cu,
// wigner.cpp:119-176, defines.h:115-210): parameter derivation, device
// buffers, the ground-state loop, ensemble initialisation, the split-step
// loop and the observables. All state lives in a bec_ctx; errors return
// status codes; host arrays belong to the caller.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "engine.h"
#include "twiddle_fp32.h"

namespace {

const double kHbar = 1.054571628e-34;   // wigner.cpp:121
const double kBohr = 5.2917720859e-11;  // wigner.cpp:122

// Neumaier-compensated host accumulator
struct HSum {
    double s = 0.0, c = 0.0;
    void add(double v)
    {
        double t = s + v;
        if (std::fabs(s) >= std::fabs(v)) c += (s - t) + v; else c += (v - t) + s;
        s = t;
    }
    double value() const { return s + c; }
};

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
int ilog2(int n) { int r = 0; while ((1 << r) < n) ++r; return r; }

struct GroupRec {
    bec_params p;
    bec_derived d;
    GeomD gd;
    GroupParamsF gf;
    int cls = -1;             // grid class (batched path)
    int traj_first = 0;       // global trajectory index of the first trajectory
    int local_first = 0;      // index within the class
    double2 *a = nullptr, *b = nullptr;   // plain path: k-space state [ne][cells]
    double2 *gs_dev = nullptr;            // batched path: x-space ground state (in the context's gs_stage)
    bool initialised = false;
};

// the pencil kernels of the per-pass schedule: register (fused_passes.cu k_pencil), persistent TMA
// (pencil_tma.cu)
constexpr int kPencilRegister = 0, kPencilTma = 1, kPencilKinds = 2;
const char *const kPencilNames[kPencilKinds] = {"register", "tma"};

struct ClassRec {
    ClassGeom geom{};
    float4 *state = nullptr;
    int *d_tgroup = nullptr, *d_tlocal = nullptr;
    double *d_traj_scale = nullptr;
    double *obs_partial = nullptr;
    double *traj_axial = nullptr;
    int tiles = 1;            // tiles per trajectory of the generic z pass
    int obs_tiles = 1;        // tiles of the pass that last wrote obs_partial
    int traj_offset = 0;      // global index of the class's first trajectory
    std::vector<int> groups;  // group indices in this class
    float2 *kin_tab[2] = {nullptr, nullptr};   // kinetic phase tables for kick fractions 0.5 and 1 (register pencils)
    int pencil_kind = 0;      // the tuned per-pass schedules' pencil kernel for this class (kPencilRegister ...)
    double pencil_ms[2] = {-1.0, -1.0};        // autotuner: ms per launch of each pencil kernel
    bool onchip = false;      // the tuned schedules run this class's steady steps as one on-chip launch
    double plane_ms = -1.0, onchip_ms = -1.0;  // autotuner: its plane launch, its on-chip step
};

} // namespace

struct bec_ctx {
    int path = 0;
    int n_traj = 0;
    std::vector<GroupRec> groups;
    std::vector<ClassRec> classes;
    std::map<int, double2 *> tw64;
    std::map<int, float2 *> tw32;
    std::map<int, float2 *> tw32_full;
    std::map<int, float2 *> tw32_nearest;
    bool use_fast = true;                // register-resident passes where the shape allows
    uint32_t *d_step = nullptr;          // batched: Philox step index the plane passes read
    bool use_graphs = true;              // batched: steady steps replay captured CUDA graphs
    bool graphs_failed = false;
    StepPlan plan;                       // batched: the fused step of the register-path classes
    std::vector<char> fused;             // per class: 1 when its passes run in the fused step
    int plan_mode = -2;                  // -2: not chosen yet, else the schedule candidate (ensure_plan)
    int plane_occupancy = 0;             // per-pass plane launches: 0 = 16 warps per SM, 1 = 20
    bool pencil_tuned = false;           // per-pass pencil launches: each class's own pencil kernel (pencil_kind)
    bool step_onchip = false;            // the step being launched is steady: classes with `onchip` take one launch
    int *d_pflags = nullptr;             // batched: [0] error flag of the TMA pencil pass, [1] a flag nothing sets,
                                         // [2] CTAs finished in the plane launch that advances the step index
    std::string plan_desc;               // the chosen plan and the autotuner's timings (JSON)
    cudaGraphExec_t step_graph[2] = {nullptr, nullptr};   // kGraphSteps steps, 1 step
    long long graph_kernels[2] = {0, 0};                  // kernels per replay of each
    GroupParamsF *d_gparams = nullptr;
    const void **d_gs_ptrs = nullptr;   // batched: device ground-state pointer of every group (bec_init_groups)
    std::vector<const void *> gs_ptrs_host;   // the table last copied to d_gs_ptrs
    char *gs_stage = nullptr;            // batched: ground states of an init call, in group order (16 B per cell)
    double *d_traj_tot = nullptr;        // [n_traj][4]
    double *d_group_mom = nullptr;       // [n_groups][4]
    int *d_group_first = nullptr, *d_group_count = nullptr;
    double *d_red = nullptr;             // reduction scratch
    double *d_scal = nullptr;            // device scalars
    double *d_plain_obs = nullptr;       // plain path per-trajectory per-z sums [n_traj][nzmax][4]
    double *d_plain_axial = nullptr;     // [n_traj][nzmax][4]
    double2 *scratch_a = nullptr, *scratch_b = nullptr;  // plain: x-space copies (max cells)
    float4 *scratch4 = nullptr;          // batched: one trajectory (max cells)
    int max_cells = 0, max_nz = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ev_h2d = nullptr;        // after an init call's copies from the caller's host arrays
    std::string err;
    long long step = 0;         // steps since initialisation (Philox counter)
    long long evo_steps = 0;    // steps since bec_start_evolution
    bool pending = false;       // batched: last step's second half-kick not yet applied
    bool has_pulse = false;     // batched: pulse waiting for the next z pass
    double2 pulse[4];           // pending pulse matrix (row-major)
    double last_ms = 0.0;
    long long last_launches = 0;
    std::vector<void *> allocs;
    size_t alloc_bytes = 0;              // bytes of the context's own device buffers
    size_t alloc_limit = 0;              // BEC_DEVICE_BYTES_LIMIT at creation (0: none)
    std::vector<WsTable> ws_tables;      // warm-start bases installed per grid
};

namespace {

bec_status fail(bec_ctx *c, bec_status st, const std::string &msg)
{
    if (c) c->err = msg;
    return st;
}

#define CKC(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? BEC_ERR_OUT_OF_MEMORY : BEC_ERR_CUDA, \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                       \
    } while (0)

#define CKL()                                                                                       \
    do {                                                                                            \
        cudaError_t e_ = cudaGetLastError();                                                        \
        if (e_ != cudaSuccess)                                                                      \
            return fail(ctx, BEC_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
    } while (0)

// A context's device buffers. With a byte limit set (BEC_DEVICE_BYTES_LIMIT), a buffer that would take the
// context past it fails as an out-of-memory allocation without reaching the device: the host-side way to
// exercise the out-of-memory paths.
template <typename T>
cudaError_t dalloc(bec_ctx *ctx, T **p, size_t n)
{
    void *q = nullptr;
    const size_t bytes = n * sizeof(T) > 0 ? n * sizeof(T) : 16;
    if (ctx->alloc_limit && ctx->alloc_bytes + bytes > ctx->alloc_limit) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e == cudaSuccess) {
        ctx->allocs.push_back(q);
        ctx->alloc_bytes += bytes;
        *p = static_cast<T *>(q);
    }
    return e;
}

double2 cd(double re, double im) { return make_double2(re, im); }

// report.tex rotation matrix: [[cos t/2, -i e^{-i phi} sin t/2], [-i e^{i phi} sin t/2, cos t/2]]
void rotation(double theta, double phi, double2 m[4])
{
    const double c = std::cos(theta / 2.0), s = std::sin(theta / 2.0);
    m[0] = cd(c, 0.0);
    m[1] = cd(-s * std::sin(phi), -s * std::cos(phi));   // -i e^{-i phi} s
    m[2] = cd(s * std::sin(phi), -s * std::cos(phi));    // -i e^{+i phi} s
    m[3] = cd(c, 0.0);
}

void matmul2(const double2 a[4], const double2 b[4], double2 out[4])
{
    auto mul = [](double2 x, double2 y) { return cd(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x); };
    auto add = [](double2 x, double2 y) { return cd(x.x + y.x, x.y + y.y); };
    double2 r[4];
    r[0] = add(mul(a[0], b[0]), mul(a[1], b[2]));
    r[1] = add(mul(a[0], b[1]), mul(a[1], b[3]));
    r[2] = add(mul(a[2], b[0]), mul(a[3], b[2]));
    r[3] = add(mul(a[2], b[1]), mul(a[3], b[3]));
    for (int i = 0; i < 4; ++i) out[i] = r[i];
}

GeomD make_geomd(const bec_params &p, const bec_derived &d)
{
    GeomD g{};
    g.nx = d.nvx; g.ny = d.nvy; g.nz = d.nvz;
    g.lx = ilog2(d.nvx); g.ly = ilog2(d.nvy); g.lz = ilog2(d.nvz);
    g.cells = d.cells;
    g.dkx = d.dkx; g.dky = d.dky; g.dkz = d.dkz;
    g.xmax = d.xmax; g.ymax = d.ymax; g.zmax = d.zmax;
    g.dx = d.dx; g.dy = d.dy; g.dz = d.dz; g.lambda = d.lambda;
    g.g11 = d.g11; g.g12 = d.g12; g.g22 = d.g22;
    g.l111 = d.l111; g.l12 = d.l12; g.l22 = d.l22; g.detuning = d.detuning;
    g.dt_evo = d.dt_evo; g.dt_steady = d.dt_steady; g.dV = d.dV;
    g.Va = d.Va; g.Vb = d.Vb;
    g.itmax = d.itmax;
    g.noise = (p.loss_noise && (d.l111 > 0 || d.l12 > 0 || d.l22 > 0)) ? 1 : 0;
    g.seed = p.seed;
    return g;
}

GroupParamsF make_gf(const GeomD &g)
{
    GroupParamsF f{};
    f.dkx = (float)g.dkx; f.dky = (float)g.dky; f.dkz = (float)g.dkz;
    f.xmax = (float)g.xmax; f.ymax = (float)g.ymax; f.zmax = (float)g.zmax;
    f.dx = (float)g.dx; f.dy = (float)g.dy; f.dz = (float)g.dz;
    f.inv_lambda2 = (float)(1.0 / (g.lambda * g.lambda));
    f.g11 = (float)g.g11; f.g12 = (float)g.g12; f.g22 = (float)g.g22;
    f.l111 = (float)g.l111; f.l12 = (float)g.l12; f.l22 = (float)g.l22;
    f.detuning = (float)g.detuning;
    f.dt = (float)g.dt_evo;
    f.noise_amp = (float)std::sqrt(g.dt_evo / (2.0 * g.dV));
    f.c1 = (float)(std::sqrt(g.l111 / 6.0) * 3.0);
    f.c2 = (float)std::sqrt(g.l12 / 2.0);
    f.c3 = (float)std::sqrt(g.l22);
    f.init_a = (float)(g.Va / std::sqrt(g.dV));
    f.init_b = (float)(g.Vb / std::sqrt(g.dV));
    f.itmax = g.itmax;
    f.noise = g.noise;
    f.seed_lo = (uint32_t)g.seed;
    f.seed_hi = (uint32_t)(g.seed >> 32);
    f.kin_x = 0.5 * g.dkx * g.dkx * g.dt_evo / (2.0 * M_PI);
    f.kin_y = g.ny > 1 ? 0.5 * g.dky * g.dky * g.dt_evo / (2.0 * M_PI) : 0.0;
    f.kin_z = 0.5 * g.dkz * g.dkz * g.dt_evo / (2.0 * M_PI);
    return f;
}

// W_n^k = exp(-2 pi i k / n), k < n/2, in double
std::vector<double2> twiddles(int n)
{
    std::vector<double2> t(n / 2 > 0 ? n / 2 : 1);
    for (int k = 0; k < n / 2; ++k) {
        double a = 2.0 * M_PI * (double)k / (double)n;
        t[k] = cd(std::cos(a), -std::sin(a));
    }
    if (n / 2 == 0) t[0] = cd(1.0, 0.0);
    return t;
}

bec_status get_tw64(bec_ctx *ctx, int n, double2 **out)
{
    auto it = ctx->tw64.find(n);
    if (it != ctx->tw64.end()) { *out = it->second; return BEC_OK; }
    std::vector<double2> t = twiddles(n);
    double2 *d = nullptr;
    CKC(dalloc(ctx, &d, t.size()));
    CKC(cudaMemcpyAsync(d, t.data(), t.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
    ctx->tw64[n] = d;
    *out = d;
    return BEC_OK;
}

// W_n^k = e^{-2 pi i k / n} in FP32: exact at multiples of a quarter turn, elsewhere the pair of modulus
// closest to 1 (twiddle_fp32.h)
float2 tw32_unit(int k, int n)
{
    k %= n;
    if ((4 * k) % n == 0) {
        const int q = 4 * k / n;
        return q == 0 ? make_float2(1.f, 0.f) : q == 1 ? make_float2(0.f, -1.f) : q == 2 ? make_float2(-1.f, 0.f)
                                                                                    : make_float2(0.f, 1.f);
    }
    const double a = 2.0 * M_PI * (double)k / (double)n;
    const fftreg::Twid t = fftreg::unit_cs(std::cos(a), -std::sin(a));
    return make_float2(t.a, t.b);
}

bec_status get_tw32(bec_ctx *ctx, int n, float2 **out)
{
    auto it = ctx->tw32.find(n);
    if (it != ctx->tw32.end()) { *out = it->second; return BEC_OK; }
    std::vector<float2> f(n / 2 > 0 ? n / 2 : 1, make_float2(1.f, 0.f));
    for (int k = 0; k < n / 2; ++k) f[k] = tw32_unit(k, n);
    float2 *d = nullptr;
    CKC(dalloc(ctx, &d, f.size()));
    CKC(cudaMemcpyAsync(d, f.data(), f.size() * sizeof(float2), cudaMemcpyHostToDevice, ctx->stream));
    ctx->tw32[n] = d;
    *out = d;
    return BEC_OK;
}

// all n twiddles W_n^e, e < n (the pencil pass indexes products j * k1 < n)
bec_status get_tw32_full(bec_ctx *ctx, int n, float2 **out)
{
    auto it = ctx->tw32_full.find(n);
    if (it != ctx->tw32_full.end()) { *out = it->second; return BEC_OK; }
    std::vector<float2> f(n);
    for (int k = 0; k < n; ++k) f[k] = tw32_unit(k, n);
    float2 *d = nullptr;
    CKC(dalloc(ctx, &d, f.size()));
    CKC(cudaMemcpyAsync(d, f.data(), f.size() * sizeof(float2), cudaMemcpyHostToDevice, ctx->stream));
    ctx->tw32_full[n] = d;
    *out = d;
    return BEC_OK;
}

// W_n^e, e < n, rounded to the nearest FP32 values (the imaginary-time passes; see tw32_unit)
bec_status get_tw32_full_nearest(bec_ctx *ctx, int n, float2 **out)
{
    auto it = ctx->tw32_nearest.find(n);
    if (it != ctx->tw32_nearest.end()) { *out = it->second; return BEC_OK; }
    std::vector<float2> f(n);
    for (int k = 0; k < n; ++k) {
        const double a = 2.0 * M_PI * (double)k / (double)n;
        f[k] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
    float2 *d = nullptr;
    CKC(dalloc(ctx, &d, f.size()));
    CKC(cudaMemcpyAsync(d, f.data(), f.size() * sizeof(float2), cudaMemcpyHostToDevice, ctx->stream));
    ctx->tw32_nearest[n] = d;
    *out = d;
    return BEC_OK;
}

bec_status plain_fft(bec_ctx *ctx, double2 *data, const GeomD &g, int inv)
{
    double2 *tx, *ty, *tz;
    bec_status st;
    if ((st = get_tw64(ctx, g.nx, &tx))) return st;
    if ((st = get_tw64(ctx, g.ny, &ty))) return st;
    if ((st = get_tw64(ctx, g.nz, &tz))) return st;
    plain_fft3d(data, g, tx, ty, tz, inv, ctx->stream);
    return BEC_OK;
}

// ---------------------------------------------------------------- plain step
// propagate (wigner.cu:178-199) for one trajectory
bec_status plain_step(bec_ctx *ctx, GroupRec &gr, int t)
{
    const GeomD &g = gr.gd;
    double2 *a = gr.a + (size_t)t * g.cells, *b = gr.b + (size_t)t * g.cells;
    bec_status st;
    plain_kick(a, b, g, 1.0, 0, ctx->stream);
    if ((st = plain_fft(ctx, a, g, 0))) return st;
    if ((st = plain_fft(ctx, b, g, 0))) return st;
    plain_nl(a, b, g, (uint32_t)t, (uint32_t)ctx->step, ctx->stream);
    if ((st = plain_fft(ctx, a, g, 1))) return st;
    if ((st = plain_fft(ctx, b, g, 1))) return st;
    plain_kick(a, b, g, 1.0 / g.cells, 1, ctx->stream);
    return BEC_OK;
}

// ---------------------------------------------------------------- batched z pass
// ends_step: no plane pass follows, so the pass leaves the state in the form a z pass reads
// ev (optional): per class (start, stop) events recorded around that class's launch
// skip_fused: leave out the classes of the fused step plan (their pencil pass runs inside it)
// a class whose steady step runs as one on-chip launch in the step being launched
bool onchip_now(const bec_ctx *ctx, const ClassRec &c)
{
    return ctx->step_onchip && ctx->pencil_tuned && c.onchip && c.kin_tab[1] && fp32_onchip_supported(c.geom);
}

bec_status batched_zpass_all(bec_ctx *ctx, float pre, float post, bool observe, const double2 *m2,
                             bool ends_step = false, std::pair<cudaEvent_t, cudaEvent_t> *ev = nullptr,
                             bool skip_fused = false)
{
    ZPassArgs z{};
    z.pre = pre;
    z.post = post;
    z.observe = observe ? 1 : 0;
    if (ctx->has_pulse) {
        z.has_m1 = 1;
        for (int i = 0; i < 4; ++i) z.m1[i] = make_float2((float)ctx->pulse[i].x, (float)ctx->pulse[i].y);
    }
    if (m2) {
        z.has_m2 = 1;
        for (int i = 0; i < 4; ++i) z.m2[i] = make_float2((float)m2[i].x, (float)m2[i].y);
    }
    // without an observation the two pulse matrices collapse into one
    float2 mfused[4];
    const float2 *mf = nullptr;
    if ((!observe && (z.has_m1 || z.has_m2)) || (observe && z.has_m1 && !z.has_m2)) {
        double2 a[4], b[4], r[4];
        for (int i = 0; i < 4; ++i) {
            a[i] = z.has_m2 ? m2[i] : cd(i == 0 || i == 3 ? 1.0 : 0.0, 0.0);
            b[i] = z.has_m1 ? ctx->pulse[i] : cd(i == 0 || i == 3 ? 1.0 : 0.0, 0.0);
        }
        matmul2(a, b, r);
        for (int i = 0; i < 4; ++i) mfused[i] = make_float2((float)r[i].x, (float)r[i].y);
        mf = mfused;
    }
    for (auto &c : ctx->classes) {
        if (c.geom.n_traj == 0) continue;
        if (skip_fused && ctx->fused[&c - &ctx->classes[0]]) continue;
        if (onchip_now(ctx, c)) continue;           // its plane-pass slot runs the whole step
        bec_status st;
        z.scale = (float)(1.0 / (double)c.geom.cells);
        z.out_scale = ends_step ? (float)(c.geom.nx * c.geom.ny) : 1.0f;
        const size_t ci = &c - &ctx->classes[0];
        if (ev) CKC(cudaEventRecord(ev[ci].first, ctx->stream));
        // the register pencil pass observes only when it also ends the step (post = 0), and kicks by the
        // fractions its kinetic tables hold (0.5, 1) or not at all
        const float kf = pre + post;
        const bool fast = ctx->use_fast && fp32_fast_pencil_supported(c.geom) &&
                          (kf == 0.0f || kf == 0.5f || kf == 1.0f) &&
                          (!observe || (post == 0.0f && ends_step && !z.has_m2));
        if (fast) {
            float2 *twf;
            if ((st = get_tw32_full(ctx, c.geom.nz, &twf))) return st;
            const float frac = kf;
            const float2 *kin = frac == 1.0f ? c.kin_tab[1] : frac == 0.5f ? c.kin_tab[0] : nullptr;
            const int kind = !observe && ctx->pencil_tuned ? c.pencil_kind : kPencilRegister;
            if (kind == kPencilTma && fp32_pencil_tma_supported(c.geom))
                CKC(fp32_pencil_tma(c.state, c.geom, twf, frac, z.scale * z.out_scale, mf, kin, ctx->d_pflags,
                                    ctx->d_pflags + 1, ctx->stream));
            else
                fp32_pencil_fast(c.state, c.geom, ctx->d_gparams, c.d_tgroup, twf, frac, z.scale * z.out_scale,
                                 mf, observe ? c.obs_partial : nullptr, z.out_scale, kin, ctx->stream);
            if (observe) c.obs_tiles = fp32_fast_pencil_tiles(c.geom);
        } else {
            float2 *tz;
            if ((st = get_tw32(ctx, c.geom.nz, &tz))) return st;
            fp32_zpass(c.state, c.geom, ctx->d_gparams, c.d_tgroup, tz, z, c.obs_partial, ctx->stream);
            if (observe) c.obs_tiles = c.tiles;
        }
        if (ev) CKC(cudaEventRecord(ev[ci].second, ctx->stream));
        CKL();
    }
    ctx->has_pulse = false;
    return BEC_OK;
}

// put_step: write ctx->step into the device step scalar first (eager launches; a captured step graph
// leaves it to the step before); skip_fused: leave out the classes of the fused step plan. advanced != NULL:
// the step index is advanced in the same pass where a class can carry it -- the register-path plane launch
// with the fewest CTAs (at most kMaxCarrierCtas, one atomic each) runs last and its last CTA increments the
// index -- and *advanced tells the caller whether that happened.
constexpr int kMaxCarrierCtas = 16384;

bec_status batched_ppass_all(bec_ctx *ctx, std::pair<cudaEvent_t, cudaEvent_t> *ev = nullptr, bool put_step = true,
                             bool skip_fused = false, bool *advanced = nullptr)
{
    if (put_step) {
        fp32_put_step(ctx->d_step, (uint32_t)ctx->step, ctx->stream);
        CKL();
    }
    const int nc = (int)ctx->classes.size();
    auto launched = [&](int ci) {
        const ClassRec &c = ctx->classes[ci];
        return c.geom.n_traj > 0 && !(skip_fused && ctx->fused[ci]);
    };
    auto onchip = [&](int ci) { return onchip_now(ctx, ctx->classes[ci]); };
    auto fast = [&](int ci) { return onchip(ci) || (ctx->use_fast && fp32_fast_plane_supported(ctx->classes[ci].geom)); };
    auto ctas = [&](int ci) {
        return onchip(ci) ? ctx->classes[ci].geom.n_traj : fp32_plane_fast_ctas(ctx->classes[ci].geom);
    };
    int carrier = -1;
    if (advanced) {
        for (int ci = 0; ci < nc; ++ci)
            if (launched(ci) && fast(ci) && ctas(ci) <= kMaxCarrierCtas && (carrier < 0 || ctas(ci) < ctas(carrier)))
                carrier = ci;
        *advanced = carrier >= 0;
    }
    for (int k = 0; k < nc; ++k) {
        // the carrier, if any, goes last
        const int ci = carrier < 0 ? k : (k < carrier ? k : k + 1 < nc ? k + 1 : carrier);
        if (!launched(ci)) continue;
        ClassRec &c = ctx->classes[ci];
        if (ev) CKC(cudaEventRecord(ev[ci].first, ctx->stream));
        if (onchip(ci)) {
            float2 *twf;
            bec_status st;
            if ((st = get_tw32_full(ctx, c.geom.nz, &twf))) return st;
            fp32_onchip_step(c.state, c.geom, ctx->d_gparams, c.d_tgroup, c.d_tlocal, twf, c.kin_tab[1], ctx->d_step,
                             ci == carrier ? ctx->d_pflags + 2 : nullptr, ctx->stream);
        } else if (fast(ci)) {
            fp32_plane_fast(c.state, c.geom, ctx->d_gparams, c.d_tgroup, c.d_tlocal, ctx->d_step, ctx->plane_occupancy,
                            ci == carrier ? ctx->d_pflags + 2 : nullptr, ctx->stream);
        } else {
            float2 *tx, *ty;
            bec_status st;
            if ((st = get_tw32(ctx, c.geom.nx, &tx))) return st;
            if ((st = get_tw32(ctx, c.geom.ny, &ty))) return st;
            fp32_ppass(c.state, c.geom, ctx->d_gparams, c.d_tgroup, c.d_tlocal, tx, ty, ctx->d_step, ctx->stream);
        }
        if (ev) CKC(cudaEventRecord(ev[ci].second, ctx->stream));
        CKL();
    }
    return BEC_OK;
}

// One split step of every class, ending with its plane pass: kick fraction pre of dt before this step's half
// kick (0.5 while the previous step's second half kick is pending), then any pending pulse. The classes of
// the fused plan run as one launch of the fused step kernel, which advances the device step index; the
// others launch their own passes, and without a fused plan the smallest plane launch advances it (or, when
// no class can carry it, a one-thread launch). put_step writes
// the host step index to the device first (eager steps); a captured step graph leaves it to the step before.
bec_status batched_step(bec_ctx *ctx, float pre, bool put_step)
{
    if (put_step) {
        fp32_put_step(ctx->d_step, (uint32_t)ctx->step, ctx->stream);
        CKL();
    }
    const bool fused = ctx->plan.ready;
    float2 mf[4];
    const bool has_m = ctx->has_pulse;
    if (has_m)
        for (int i = 0; i < 4; ++i) mf[i] = make_float2((float)ctx->pulse[i].x, (float)ctx->pulse[i].y);
    bec_status st;
    // a steady step (the previous step's second half kick pending, no pulse): the on-chip classes take one launch
    ctx->step_onchip = !fused && pre == 0.5f && !has_m;
    struct Clear { bool &f; ~Clear() { f = false; } } clear{ctx->step_onchip};
    if ((st = batched_zpass_all(ctx, pre, 0.5f, false, nullptr, false, nullptr, fused))) return st;
    bool advanced = false;
    if ((st = batched_ppass_all(ctx, nullptr, false, fused, fused ? nullptr : &advanced))) return st;
    if (fused) step_launch(ctx->plan, ctx->d_gparams, ctx->d_step, pre + 0.5f, has_m ? mf : nullptr, ctx->stream);
    else if (!advanced) fp32_inc_step(ctx->d_step, ctx->stream);
    CKL();
    return BEC_OK;
}

// The split-step schedule of a batched context, chosen once before its first step. Candidates:
//   0  per-pass launches, plane passes at 16 warps per SM (no register spill)
//   1  per-pass launches, plane passes at 20 warps per SM (96 registers, a small spill)
//   2, 3  as 0, 1 with each class's non-observing pencil pass on the faster pencil kernel (pick_pencil_kernels)
//   4 + k  the fused step kernel on work list k (two-phase, interleaved at 0.5, 1, 2, 4 waves)
// BEC_STEP_PLAN in the environment forces one ("unfused" = 0, "unfused-20" = 1, "unfused-tma" = 2 and
// "unfused-20-tma" = 3 with every class on the TMA pencil kernel, "0".."4" = fused k); otherwise a choice
// cached for the same class mix on this device is reused, or every candidate is timed on a copy of the state
// (BEC_AUTOTUNE=0 skips the timing and takes candidate 0).
constexpr int kPerPassCandidates = 4;
constexpr int kAllCandidates = kPerPassCandidates + kStepCandidates;
const char *const kPerPassNames[kPerPassCandidates] = {"unfused", "unfused-20", "unfused-tma", "unfused-20-tma"};
constexpr size_t kPickClasses = 11;   // classes whose picks the plan cache keeps (two bits each above bit 8)

std::string candidate_name(int c)
{
    if (c < kPerPassCandidates)
        return std::string("per-pass launches, ") + (c & 1 ? "20" : "16") + " warps per SM" +
               (c >= 2 ? ", pencil kernel tuned per class" : "");
    return std::string("fused ") + step_plan_name(c - kPerPassCandidates);
}

bec_status check_step_error(bec_ctx *ctx);

// Per grid class, the faster of the two pencil kernels for the full-kick pass of a steady step: the register
// kernel (16 pencils per CTA of nz threads, 16 warps per SM) or the persistent TMA kernel (three CTAs per SM,
// the next tile's load in flight). Both compute the same bits; each is timed over three launches after one
// warm-up on the current state (the caller restores it).
bec_status pick_pencil_kernels(bec_ctx *ctx)
{
    for (auto &c : ctx->classes) {
        c.pencil_kind = kPencilRegister;
        c.pencil_ms[0] = c.pencil_ms[1] = -1.0;
        c.onchip = false;
        c.plane_ms = c.onchip_ms = -1.0;
        if (c.geom.n_traj == 0 || !ctx->use_fast || !fp32_fast_pencil_supported(c.geom) || !c.kin_tab[1]) continue;
        float2 *twf;
        bec_status st;
        if ((st = get_tw32_full(ctx, c.geom.nz, &twf))) return st;
        const float scale = (float)(1.0 / (double)c.geom.cells);
        for (int kind = 0; kind < kPencilKinds; ++kind) {
            if (kind == kPencilTma && !fp32_pencil_tma_supported(c.geom)) continue;
            for (int r = 0; r < 4; ++r) {
                if (r == 1) CKC(cudaEventRecord(ctx->ev0, ctx->stream));
                if (kind == kPencilRegister)
                    fp32_pencil_fast(c.state, c.geom, ctx->d_gparams, c.d_tgroup, twf, 1.0f, scale, nullptr, nullptr,
                                     1.0f, c.kin_tab[1], ctx->stream);
                else
                    CKC(fp32_pencil_tma(c.state, c.geom, twf, 1.0f, scale, nullptr, c.kin_tab[1], ctx->d_pflags,
                                        ctx->d_pflags + 1, ctx->stream));
            }
            CKC(cudaEventRecord(ctx->ev1, ctx->stream));
            CKC(cudaEventSynchronize(ctx->ev1));
            float ms = 0.f;
            CKC(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
            c.pencil_ms[kind] = ms / 3.0;
            if (c.pencil_ms[kind] < c.pencil_ms[c.pencil_kind]) c.pencil_kind = kind;
        }
        // an 8x8x64 class: its steady step as one on-chip launch against its faster pencil launch plus its plane
        // launch (the step index is left alone: no launch here advances it)
        if (fp32_onchip_supported(c.geom) && fp32_fast_plane_supported(c.geom)) {
            for (int kind = 0; kind < 2; ++kind) {
                for (int r = 0; r < 4; ++r) {
                    if (r == 1) CKC(cudaEventRecord(ctx->ev0, ctx->stream));
                    if (kind == 0)
                        fp32_plane_fast(c.state, c.geom, ctx->d_gparams, c.d_tgroup, c.d_tlocal, ctx->d_step,
                                        ctx->plane_occupancy, nullptr, ctx->stream);
                    else
                        fp32_onchip_step(c.state, c.geom, ctx->d_gparams, c.d_tgroup, c.d_tlocal, twf, c.kin_tab[1],
                                         ctx->d_step, nullptr, ctx->stream);
                }
                CKC(cudaEventRecord(ctx->ev1, ctx->stream));
                CKC(cudaEventSynchronize(ctx->ev1));
                float ms = 0.f;
                CKC(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
                (kind == 0 ? c.plane_ms : c.onchip_ms) = ms / 3.0;
            }
            c.onchip = c.onchip_ms < c.pencil_ms[c.pencil_kind] + c.plane_ms;
        }
    }
    return BEC_OK;
}

bec_status ensure_plan(bec_ctx *ctx)
{
    if (ctx->path != BEC_PATH_FP32_BATCHED || ctx->plan_mode != -2) return BEC_OK;
    ctx->fused.assign(ctx->classes.size(), 0);
    const char *force = std::getenv("BEC_STEP_PLAN");
    const std::string fs = force ? force : "";
    std::vector<ClassGeom> geoms;
    std::vector<StepClassDev> devs;
    std::vector<int> offs, idx;
    if (ctx->use_fast) {
        for (size_t ci = 0; ci < ctx->classes.size(); ++ci) {
            ClassRec &c = ctx->classes[ci];
            if (c.geom.n_traj == 0 || !step_class_supported(c.geom)) continue;
            float2 *twf;
            bec_status st;
            if ((st = get_tw32_full(ctx, c.geom.nz, &twf))) return st;
            StepClassDev d{};
            d.state = c.state;
            d.tgroup = c.d_tgroup;
            d.tlocal = c.d_tlocal;
            d.tw = twf;
            d.nx = c.geom.nx; d.ny = c.geom.ny; d.nz = c.geom.nz; d.lx = c.geom.lx;
            d.cells = c.geom.cells; d.tiles = c.geom.nx * c.geom.ny / 16; d.n_traj = c.geom.n_traj;
            d.kin[0] = c.kin_tab[0];
            d.kin[1] = c.kin_tab[1];
            geoms.push_back(c.geom);
            devs.push_back(d);
            offs.push_back(c.traj_offset);
            idx.push_back((int)ci);
        }
    }
    // schedule c: per-pass occupancy / fused work list, no timing
    auto apply = [&](int c) -> bec_status {
        if (c < kPerPassCandidates) {
            ctx->plan.ready = false;
            ctx->plane_occupancy = c & 1;
            ctx->pencil_tuned = c >= 2;
            for (int ci : idx) ctx->fused[ci] = 0;
            return BEC_OK;
        }
        if (step_plan_build(ctx->plan, geoms, devs, offs, c - kPerPassCandidates, ctx->stream) != cudaSuccess)
            return fail(ctx, BEC_ERR_CUDA, "fused step plan");
        ctx->plane_occupancy = 0;
        ctx->pencil_tuned = false;
        for (int ci : idx) ctx->fused[ci] = 1;
        return BEC_OK;
    };
    int cand = 0;
    std::string how = "default";
    std::vector<double> tms(kAllCandidates, -1.0);
    bec_status st;
    const int named = (int)(std::find(kPerPassNames, kPerPassNames + kPerPassCandidates, fs) - kPerPassNames);
    if (named < kPerPassCandidates) {
        cand = named;                                  // "-tma": every class on the TMA pencil kernel
        for (auto &c : ctx->classes) {
            c.pencil_kind = named < 2 ? kPencilRegister : kPencilTma;
            c.onchip = false;
        }
        how = "forced";
    } else if (fs == "unfused-onchip") {
        cand = 2;                                      // register pencils, every 8x8x64 class on-chip
        for (auto &c : ctx->classes) {
            c.pencil_kind = kPencilRegister;
            c.onchip = fp32_onchip_supported(c.geom);
        }
        how = "forced";
    } else if (!fs.empty()) {
        const int k = std::atoi(fs.c_str());
        if (k < 0 || k >= kStepCandidates || geoms.empty())
            return fail(ctx, BEC_ERR_INVALID_ARG, "BEC_STEP_PLAN: no such fused work list for this context");
        cand = kPerPassCandidates + k;
        how = "forced";
    } else if (step_plan_cached(geoms, &cand)) {
        // the candidate, and above bit 8 two bits per class: its pencil kernel, its on-chip step
        for (size_t ci = 0; ci < ctx->classes.size() && ci < kPickClasses; ++ci) {
            ctx->classes[ci].pencil_kind = (cand >> (8 + 2 * ci)) & 1;
            ctx->classes[ci].onchip = (cand >> (9 + 2 * ci)) & 1;
        }
        cand &= 0xFF;
        how = "cached";
    } else {
        const char *at = std::getenv("BEC_AUTOTUNE");
        const int n_cand = geoms.empty() ? kPerPassCandidates : kAllCandidates;
        if (!(at && at[0] == '0')) {
            // time every candidate's full step on a copy of the state: the copy (and any pending pulse) is
            // restored afterwards, so tuning changes nothing of the run; every candidate computes the same bits
            size_t bytes = 0;
            for (auto &c : ctx->classes) bytes += sizeof(float4) * (size_t)c.geom.n_traj * c.geom.cells;
            char *save = nullptr;
            if (cudaMalloc(&save, bytes) == cudaSuccess) {
                size_t o = 0;
                for (auto &c : ctx->classes) {
                    const size_t n = sizeof(float4) * (size_t)c.geom.n_traj * c.geom.cells;
                    if (n) CKC(cudaMemcpyAsync(save + o, c.state, n, cudaMemcpyDeviceToDevice, ctx->stream));
                    o += n;
                }
                const bool had_pulse = ctx->has_pulse;
                ctx->has_pulse = false;
                st = pick_pencil_kernels(ctx);
                double best = 1e30;
                for (int k = 0; k < n_cand && st == BEC_OK; ++k) {
                    if ((st = apply(k))) break;
                    for (int r = 0; r < 4 && st == BEC_OK; ++r) {
                        if (r == 1) cudaEventRecord(ctx->ev0, ctx->stream);
                        st = batched_step(ctx, 0.5f, true);
                    }
                    if (st) break;
                    cudaEventRecord(ctx->ev1, ctx->stream);
                    if (cudaEventSynchronize(ctx->ev1) != cudaSuccess) {
                        st = fail(ctx, BEC_ERR_CUDA, std::string("step timing: ") + cudaGetErrorString(cudaGetLastError()));
                        break;
                    }
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
                    tms[k] = ms / 3.0;
                    if (tms[k] < best) { best = tms[k]; cand = k; }
                }
                o = 0;
                for (auto &c : ctx->classes) {
                    const size_t n = sizeof(float4) * (size_t)c.geom.n_traj * c.geom.cells;
                    if (n) cudaMemcpyAsync(c.state, save + o, n, cudaMemcpyDeviceToDevice, ctx->stream);
                    o += n;
                }
                cudaStreamSynchronize(ctx->stream);
                cudaFree(save);
                ctx->has_pulse = had_pulse;
                if (st) return st;
                if ((st = check_step_error(ctx))) return st;
                how = "autotuned";
                int picks = 0;
                for (size_t ci = 0; ci < ctx->classes.size() && ci < kPickClasses; ++ci)
                    picks |= (ctx->classes[ci].pencil_kind << (8 + 2 * ci)) |
                             ((ctx->classes[ci].onchip ? 1 : 0) << (9 + 2 * ci));
                step_plan_remember(geoms, cand | picks);
            } else {
                cudaGetLastError();
            }
        }
    }
    if ((st = apply(cand))) return st;
    CKC(cudaStreamSynchronize(ctx->stream));
    ctx->plan_mode = cand;
    const bool fused = cand >= kPerPassCandidates;
    int n_classes = 0;
    for (auto &c : ctx->classes) n_classes += c.geom.n_traj > 0;
    char buf[256];
    std::string j = "{\"plan\": \"" + candidate_name(cand) + "\", \"candidate\": " + std::to_string(cand) +
                    ", \"chosen\": \"" + how + "\", \"fused_classes\": " + std::to_string(fused ? (int)idx.size() : 0) +
                    ", \"launches_per_step\": " +
                    std::to_string(fused ? (ctx->plan.two_phase ? 2 : 1) + 2 * (n_classes - (int)idx.size())
                                         : 2 * n_classes);
    if (fused) j += ", \"grid\": " + std::to_string(ctx->plan.grid) + ", \"items\": " + std::to_string(ctx->plan.n_items);
    j += ", \"pencil_kernels\": [";
    bool firstc = true;
    for (auto &c : ctx->classes) {
        if (c.geom.n_traj == 0) continue;
        const int kind = ctx->pencil_tuned ? c.pencil_kind : kPencilRegister;
        const bool oc = ctx->pencil_tuned && c.onchip && fp32_onchip_supported(c.geom);
        std::snprintf(buf, sizeof buf,
                      "%s{\"grid\": [%d, %d, %d], \"kernel\": \"%s\", \"register_ms\": %.4f, \"tma_ms\": %.4f, "
                      "\"onchip\": %s, \"plane_ms\": %.4f, \"onchip_ms\": %.4f}",
                      firstc ? "" : ", ", c.geom.nx, c.geom.ny, c.geom.nz, kPencilNames[kind], c.pencil_ms[0],
                      c.pencil_ms[1], oc ? "true" : "false", c.plane_ms, c.onchip_ms);
        j += buf;
        firstc = false;
    }
    j += "], \"candidates\": [";
    for (int k = 0; k < kAllCandidates; ++k) j += (k ? ", \"" : "\"") + candidate_name(k) + "\"";
    j += "], \"candidate_ms_per_step\": [";
    for (int k = 0; k < kAllCandidates; ++k) {
        std::snprintf(buf, sizeof buf, "%s%.4f", k ? ", " : "", tms[k]);
        j += buf;
    }
    ctx->plan_desc = j + "]}";
    return BEC_OK;
}

// reduces the partial sums of the last observing z pass into d_traj_tot / axial / group moments
bec_status batched_reduce_obs(bec_ctx *ctx)
{
    for (auto &c : ctx->classes) {
        if (c.geom.n_traj == 0) continue;
        obs_reduce(c.obs_partial, c.geom.n_traj, c.obs_tiles, c.geom.nz, c.d_traj_scale, c.traj_axial,
                   ctx->d_traj_tot + (size_t)c.traj_offset * 4, ctx->stream);
        CKL();
    }
    group_reduce(ctx->d_traj_tot, ctx->d_group_first, ctx->d_group_count, (int)ctx->groups.size(),
                 ctx->d_group_mom, ctx->stream);
    CKL();
    return BEC_OK;
}

// Moments of the step boundary while the step's second half kick is still pending (no pulse waiting),
// without ending the step. The pending kick multiplies every k-space amplitude of both components by
// the same unit-modulus factor, so |a|^2, |b|^2 and conj(a) b summed over the trajectory are those of
// the stored state (Parseval), which is nx ny times the normalised ifft_xy representation of the
// observing z pass: the sums are scaled by 1 / (nx ny)^2 and then reduced like an observing pass.
bec_status batched_moments_stored(bec_ctx *ctx)
{
    for (auto &c : ctx->classes) {
        if (c.geom.n_traj == 0) continue;
        const int blocks = std::max(1, std::min({16, c.geom.cells / 16384, c.geom.nz}));
        const double inv = 1.0 / ((double)c.geom.nx * (double)c.geom.ny);
        fp32_state_sums(c.state, c.geom.cells, c.geom.n_traj, blocks, inv * inv, c.obs_partial, ctx->stream);
        CKL();
        obs_reduce(c.obs_partial, c.geom.n_traj, blocks, 1, c.d_traj_scale, nullptr,
                   ctx->d_traj_tot + (size_t)c.traj_offset * 4, ctx->stream);
        CKL();
    }
    group_reduce(ctx->d_traj_tot, ctx->d_group_first, ctx->d_group_count, (int)ctx->groups.size(),
                 ctx->d_group_mom, ctx->stream);
    CKL();
    return BEC_OK;
}

// Brings the batched state to a step boundary with no pending kick or pulse.
bec_status batched_resolve(bec_ctx *ctx, bool observe)
{
    if (!ctx->pending && !ctx->has_pulse && !observe) return BEC_OK;
    bec_status st = batched_zpass_all(ctx, ctx->pending ? 0.5f : 0.0f, 0.0f, observe, nullptr, true);
    if (st) return st;
    ctx->pending = false;
    return BEC_OK;
}

// Error flags of the fused step kernel (a dependency wait that gave up) and of the TMA pencil kernel (a tile
// load wait that gave up); both kernels bound every wait.
bec_status check_step_error(bec_ctx *ctx)
{
    int err = 0;
    CKC(step_read_error(ctx->plan, &err, ctx->stream));
    if (err) return fail(ctx, BEC_ERR_CUDA, "fused step: a dependency wait gave up (state of that step is invalid)");
    if (ctx->pencil_tuned && ctx->d_pflags) {
        CKC(cudaMemcpyAsync(&err, ctx->d_pflags, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CKC(cudaStreamSynchronize(ctx->stream));
        if (err) {
            CKC(cudaMemsetAsync(ctx->d_pflags, 0, sizeof(int), ctx->stream));   // reported once
            return fail(ctx, BEC_ERR_CUDA, "TMA pencil pass: a tile load wait gave up (state of that step is invalid)");
        }
    }
    return BEC_OK;
}

// ---------------------------------------------------------------- captured step loop
// A steady step (the previous step's second half-kick pending, no pulse, no observation) launches the
// same kernels with the same arguments every time: the full kick in the pencil passes, the plane passes
// (the step scalar advanced by the last CTA of the smallest one, or of the fused kernel, or by a one-thread
// launch). kGraphSteps of them, and one, are captured once per context and replayed; the device step
// scalar is set once before a stretch of replays.
constexpr int kGraphSteps = 8;

bec_status capture_steps(bec_ctx *ctx, int k, cudaGraphExec_t *out, long long *kernels)
{
    const long long l0 = g_launches;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return BEC_ERR_CUDA;
    }
    bec_status st = BEC_OK;
    for (int i = 0; i < k && st == BEC_OK; ++i) {
        st = batched_step(ctx, 0.5f, false);
    }
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    *kernels = g_launches - l0;
    g_launches = l0;                    // captured, not launched
    if (st != BEC_OK || e != cudaSuccess || !graph) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return st != BEC_OK ? st : BEC_ERR_CUDA;
    }
    const cudaError_t e2 = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) {
        *out = nullptr;
        cudaGetLastError();
        return BEC_ERR_CUDA;
    }
    return BEC_OK;
}

// m steady steps (requires ctx->pending and no pulse waiting)
bec_status run_steady(bec_ctx *ctx, long long m)
{
    if (m <= 0) return BEC_OK;
    bool graphs = ctx->use_graphs && !ctx->graphs_failed;
    if (graphs && !ctx->step_graph[0]) {
        // every buffer and twiddle table a steady step touches exists once an eager step has run
        if (capture_steps(ctx, kGraphSteps, &ctx->step_graph[0], &ctx->graph_kernels[0]) != BEC_OK ||
            capture_steps(ctx, 1, &ctx->step_graph[1], &ctx->graph_kernels[1]) != BEC_OK) {
            ctx->graphs_failed = true;
            graphs = false;
        }
    }
    if (!graphs) {
        for (long long i = 0; i < m; ++i) {
            bec_status st = batched_step(ctx, 0.5f, true);
            if (st) return st;
            ctx->step++;
            ctx->evo_steps++;
        }
        return BEC_OK;
    }
    fp32_put_step(ctx->d_step, (uint32_t)ctx->step, ctx->stream);   // each replayed step advances it at its end
    CKL();
    for (long long i = 0; i < m / kGraphSteps; ++i) {
        CKC(cudaGraphLaunch(ctx->step_graph[0], ctx->stream));
        g_launches += ctx->graph_kernels[0];
    }
    for (long long i = 0; i < m % kGraphSteps; ++i) {
        CKC(cudaGraphLaunch(ctx->step_graph[1], ctx->stream));
        g_launches += ctx->graph_kernels[1];
    }
    ctx->step += m;
    ctx->evo_steps += m;
    return BEC_OK;
}

// plain path: per-trajectory per-z sums of x-space copies, then reductions
bec_status plain_observe(bec_ctx *ctx)
{
    CKC(cudaMemsetAsync(ctx->d_plain_obs, 0, sizeof(double) * (size_t)ctx->n_traj * ctx->max_nz * 4, ctx->stream));
    for (auto &gr : ctx->groups) {
        const GeomD &g = gr.gd;
        for (int t = 0; t < gr.p.ne; ++t) {
            CKC(cudaMemcpyAsync(ctx->scratch_a, gr.a + (size_t)t * g.cells, sizeof(double2) * g.cells,
                                cudaMemcpyDeviceToDevice, ctx->stream));
            CKC(cudaMemcpyAsync(ctx->scratch_b, gr.b + (size_t)t * g.cells, sizeof(double2) * g.cells,
                                cudaMemcpyDeviceToDevice, ctx->stream));
            bec_status st;
            if ((st = plain_fft(ctx, ctx->scratch_a, g, 0))) return st;
            if ((st = plain_fft(ctx, ctx->scratch_b, g, 0))) return st;
            plain_axial_sums(ctx->scratch_a, ctx->scratch_b, g,
                             ctx->d_plain_obs + (size_t)(gr.traj_first + t) * ctx->max_nz * 4, ctx->stream);
            CKL();
        }
    }
    // the per-trajectory rows are max_nz long; groups with a shorter nz have zero tails
    obs_reduce(ctx->d_plain_obs, ctx->n_traj, 1, ctx->max_nz, nullptr, ctx->d_plain_axial, ctx->d_traj_tot,
               ctx->stream);
    CKL();
    group_reduce(ctx->d_traj_tot, ctx->d_group_first, ctx->d_group_count, (int)ctx->groups.size(),
                 ctx->d_group_mom, ctx->stream);
    CKL();
    return BEC_OK;
}

bec_status check_ready(bec_ctx *ctx)
{
    for (auto &g : ctx->groups)
        if (!g.initialised) return fail(ctx, BEC_ERR_STATE, "every group needs bec_init_group first");
    return BEC_OK;
}

bec_status do_evolve(bec_ctx *ctx, int n)
{
    bec_status st;
    if (ctx->path == BEC_PATH_FP64_PLAIN) {
        for (int s = 0; s < n; ++s) {
            for (auto &gr : ctx->groups)
                for (int t = 0; t < gr.p.ne; ++t)
                    if ((st = plain_step(ctx, gr, t))) return st;
            CKL();
            ctx->step++;
            ctx->evo_steps++;
        }
    } else {
        int s = 0;
        if ((st = ensure_plan(ctx))) return st;
        if (n > 0 && (!ctx->pending || ctx->has_pulse)) {      // an eager first step starts the stretch
            if ((st = batched_step(ctx, ctx->pending ? 0.5f : 0.0f, true))) return st;
            ctx->pending = true;
            ctx->step++;
            ctx->evo_steps++;
            s = 1;
        }
        if ((st = run_steady(ctx, n - s))) return st;
    }
    return BEC_OK;
}

bec_status apply_pulse(bec_ctx *ctx, const double2 m[4])
{
    if (ctx->path == BEC_PATH_FP64_PLAIN) {
        for (auto &gr : ctx->groups) {
            plain_pulse(gr.a, gr.b, gr.p.ne * gr.gd.cells, m[0], m[1], m[2], m[3], ctx->stream);
            CKL();
        }
    } else {
        if (ctx->has_pulse) {
            double2 r[4];
            matmul2(m, ctx->pulse, r);
            for (int i = 0; i < 4; ++i) ctx->pulse[i] = r[i];
        } else {
            for (int i = 0; i < 4; ++i) ctx->pulse[i] = m[i];
        }
        ctx->has_pulse = true;
    }
    return BEC_OK;
}

bec_status fetch_group_moments(bec_ctx *ctx, bec_moments *out)
{
    const size_t ng = ctx->groups.size();
    std::vector<double> h(ng * 4);
    CKC(cudaMemcpyAsync(h.data(), ctx->d_group_mom, sizeof(double) * ng * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CKC(cudaStreamSynchronize(ctx->stream));
    for (size_t g = 0; g < ng; ++g) {
        out[g].t = ctx->evo_steps * ctx->groups[g].p.dt_evo;
        out[g].na = h[g * 4 + 0];
        out[g].nb = h[g * 4 + 1];
        out[g].s_re = h[g * 4 + 2];
        out[g].s_im = h[g * 4 + 3];
        if (!std::isfinite(out[g].na) || !std::isfinite(out[g].nb) || !std::isfinite(out[g].s_re) ||
            !std::isfinite(out[g].s_im))
            return fail(ctx, BEC_ERR_NUMERICAL, "non-finite moments (state diverged)");
    }
    return BEC_OK;
}

bec_status observe_now(bec_ctx *ctx)
{
    if (ctx->path == BEC_PATH_FP64_PLAIN) return plain_observe(ctx);
    bec_status st = batched_resolve(ctx, true);
    if (st) return st;
    return batched_reduce_obs(ctx);
}

} // namespace

// ============================================================================ C ABI
extern "C" {

int32_t bec_abi_version(void) { return BEC_ABI_VERSION; }

bec_status bec_derive_params(const bec_params *p, bec_derived *d)
{
    if (!p || !d) return BEC_ERR_INVALID_ARG;
    if (!is_pow2(p->nvx) || !is_pow2(p->nvy) || !is_pow2(p->nvz) || p->nvx < 2 || p->nvz < 2)
        return BEC_ERR_UNSUPPORTED_GRID;
    if (!(p->m > 0) || !(p->fx > 0) || !(p->fz > 0) || !(p->N > 0) || p->ne < 1 || p->itmax < 1)
        return BEC_ERR_INVALID_ARG;
    std::memset(d, 0, sizeof(*d));
    const double w_rho = 2.0 * M_PI * p->fx;
    d->l_rho = std::sqrt(kHbar / (p->m * w_rho));
    d->t_rho = 1.0 / w_rho;
    d->lambda = p->fx / p->fz;
    d->nvx = p->nvx; d->nvy = p->nvy; d->nvz = p->nvz;
    d->cells = p->nvx * p->nvy * p->nvz;
    d->dims = (p->nvy == 1) ? 2 : 3;
    d->Va = p->Va; d->Vb = p->Vb;
    d->V = (p->Va + p->Vb) / 2.0;
    d->detuning = 2.0 * M_PI * p->detuning / w_rho;
    d->l111 = p->gamma111 / (std::pow(d->l_rho, 6) * w_rho);
    d->l12 = p->gamma12 / (std::pow(d->l_rho, 3) * w_rho);
    d->l22 = p->gamma22 / (std::pow(d->l_rho, 3) * w_rho);
    d->g11 = 4.0 * M_PI * p->a11 * kBohr / d->l_rho;
    d->g12 = 4.0 * M_PI * p->a12 * kBohr / d->l_rho;
    d->g22 = 4.0 * M_PI * p->a22 * kBohr / d->l_rho;
    d->N = p->N;
    if (d->dims == 3) {
        d->mu = std::pow(15.0 * d->N * d->g11 / (16.0 * M_PI * d->lambda * std::sqrt(2.0)), 0.4);
        d->xmax = 1.2 * std::sqrt(2.0 * d->mu);
        d->ymax = 1.2 * std::sqrt(2.0 * d->mu);
        d->zmax = 1.2 * d->lambda * std::sqrt(2.0 * d->mu);
        d->dx = 2.0 * d->xmax / (d->nvx - 1);
        d->dy = 2.0 * d->ymax / (d->nvy - 1);
        d->dz = 2.0 * d->zmax / (d->nvz - 1);
        d->dkx = M_PI / d->xmax;
        d->dky = M_PI / d->ymax;
        d->dkz = M_PI / d->zmax;
    } else {
        // 2D x-z slice: transverse oscillator ground state of width l_y = sqrt(hbar / m w_y);
        // couplings and two-body rates scale by 1/(sqrt(2 pi) l_y), the three-body rate by
        // 1/(sqrt(3) pi l_y^2); Thomas-Fermi N = pi lambda mu^2 / g11.
        const double ly = std::sqrt(p->fx / (p->fy > 0 ? p->fy : p->fx));
        const double s2 = 1.0 / (std::sqrt(2.0 * M_PI) * ly);
        const double s3 = 1.0 / (std::sqrt(3.0) * M_PI * ly * ly);
        d->g11 *= s2; d->g12 *= s2; d->g22 *= s2;
        d->l12 *= s2; d->l22 *= s2; d->l111 *= s3;
        d->mu = std::sqrt(d->N * d->g11 / (M_PI * d->lambda));
        d->xmax = 1.2 * std::sqrt(2.0 * d->mu);
        d->ymax = 0.0;
        d->zmax = 1.2 * d->lambda * std::sqrt(2.0 * d->mu);
        d->dx = 2.0 * d->xmax / (d->nvx - 1);
        d->dy = 1.0;
        d->dz = 2.0 * d->zmax / (d->nvz - 1);
        d->dkx = M_PI / d->xmax;
        d->dky = 0.0;
        d->dkz = M_PI / d->zmax;
    }
    d->dV = d->dx * d->dy * d->dz;
    d->itmax = p->itmax;
    d->dt_steady = p->dt_steady / d->t_rho;
    d->t_equilib = p->t_equilib / d->t_rho;
    d->dt_evo = p->dt_evo / d->t_rho;
    d->ne = p->ne;
    int n = 0;
    double t = 0.0;
    if (d->dt_evo > 0) {
        while (t <= d->t_equilib && n < 100000000) { ++n; t += d->dt_evo; }
    } else {
        n = 1;
    }
    d->n_equil_steps = n;
    return BEC_OK;
}

bec_status bec_create(const bec_params *groups, int32_t n_groups, int32_t path, bec_ctx **out)
{
    if (!out) return BEC_ERR_INVALID_ARG;
    *out = nullptr;
    if (!groups || n_groups < 1) return BEC_ERR_INVALID_ARG;
    if (path != BEC_PATH_FP64_PLAIN && path != BEC_PATH_FP32_BATCHED) return BEC_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return BEC_ERR_NO_DEVICE;
    }
    bec_ctx *ctx = new bec_ctx();
    ctx->path = path;
    if (const char *lim = std::getenv("BEC_DEVICE_BYTES_LIMIT")) ctx->alloc_limit = (size_t)std::strtoull(lim, nullptr, 10);
    ctx->groups.resize(n_groups);
    for (int g = 0; g < n_groups; ++g) {
        GroupRec &gr = ctx->groups[g];
        gr.p = groups[g];
        bec_status st = bec_derive_params(&gr.p, &gr.d);
        if (st) { delete ctx; return st; }
        if (gr.d.nvx > 1024 || gr.d.nvy > 1024 || gr.d.nvz > 1024) { delete ctx; return BEC_ERR_UNSUPPORTED_GRID; }
        if (path == BEC_PATH_FP32_BATCHED) {
            // the z pass holds whole pencils of 16 (or nvx) columns; the plane pass whole planes
            if (gr.d.nvz > 512 || gr.d.nvx * gr.d.nvy > 2048 || gr.d.nvz < 2) { delete ctx; return BEC_ERR_UNSUPPORTED_GRID; }
        }
        gr.gd = make_geomd(gr.p, gr.d);
        gr.gf = make_gf(gr.gd);
        ctx->max_cells = std::max(ctx->max_cells, gr.d.cells);
        ctx->max_nz = std::max(ctx->max_nz, gr.d.nvz);
    }
    bec_status st = BEC_OK;
    auto bail = [&](bec_status s) { bec_destroy(ctx); return s; };
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(BEC_ERR_CUDA);
    if (cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_h2d, cudaEventDisableTiming) != cudaSuccess)
        return bail(BEC_ERR_CUDA);

    // trajectory numbering: classes in first-appearance order, groups in order within a class
    if (path == BEC_PATH_FP32_BATCHED) {
        for (int g = 0; g < n_groups; ++g) {
            GroupRec &gr = ctx->groups[g];
            int cls = -1;
            for (size_t c = 0; c < ctx->classes.size(); ++c) {
                const ClassGeom &cg = ctx->classes[c].geom;
                if (cg.nx == gr.d.nvx && cg.ny == gr.d.nvy && cg.nz == gr.d.nvz) { cls = (int)c; break; }
            }
            if (cls < 0) {
                ClassRec cr;
                cr.geom.nx = gr.d.nvx; cr.geom.ny = gr.d.nvy; cr.geom.nz = gr.d.nvz;
                cr.geom.lx = ilog2(gr.d.nvx); cr.geom.ly = ilog2(gr.d.nvy); cr.geom.lz = ilog2(gr.d.nvz);
                cr.geom.cells = gr.d.cells;
                cr.geom.n_traj = 0;
                ctx->classes.push_back(cr);
                cls = (int)ctx->classes.size() - 1;
            }
            gr.cls = cls;
            ctx->classes[cls].groups.push_back(g);
        }
        int off = 0;
        for (auto &c : ctx->classes) {
            c.traj_offset = off;
            int local = 0;
            for (int g : c.groups) {
                GroupRec &gr = ctx->groups[g];
                gr.traj_first = off + local;
                gr.local_first = local;
                local += gr.p.ne;
            }
            c.geom.n_traj = local;
            off += local;
        }
        ctx->n_traj = off;
    } else {
        int off = 0;
        for (auto &gr : ctx->groups) { gr.traj_first = off; off += gr.p.ne; }
        ctx->n_traj = off;
    }
    ctx->last_launches = 0;

    // device buffers
#define CKA(call) do { if ((call) != cudaSuccess) { cudaGetLastError(); return bail(BEC_ERR_OUT_OF_MEMORY); } } while (0)
    const int ng = n_groups;
    CKA(dalloc(ctx, &ctx->d_traj_tot, (size_t)ctx->n_traj * 4));
    CKA(dalloc(ctx, &ctx->d_group_mom, (size_t)ng * 4));
    CKA(dalloc(ctx, &ctx->d_group_first, (size_t)ng));
    CKA(dalloc(ctx, &ctx->d_group_count, (size_t)ng));
    CKA(dalloc(ctx, &ctx->d_red, (size_t)2 * 8 * 1024));
    CKA(dalloc(ctx, &ctx->d_scal, (size_t)64));
    {
        std::vector<int> first(ng), count(ng);
        for (int g = 0; g < ng; ++g) { first[g] = ctx->groups[g].traj_first; count[g] = ctx->groups[g].p.ne; }
        CKA(cudaMemcpyAsync(ctx->d_group_first, first.data(), sizeof(int) * ng, cudaMemcpyHostToDevice, ctx->stream));
        CKA(cudaMemcpyAsync(ctx->d_group_count, count.data(), sizeof(int) * ng, cudaMemcpyHostToDevice, ctx->stream));
    }
    if (path == BEC_PATH_FP64_PLAIN) {
        for (auto &gr : ctx->groups) {
            CKA(dalloc(ctx, &gr.a, (size_t)gr.p.ne * gr.d.cells));
            CKA(dalloc(ctx, &gr.b, (size_t)gr.p.ne * gr.d.cells));
        }
        CKA(dalloc(ctx, &ctx->scratch_a, (size_t)ctx->max_cells));
        CKA(dalloc(ctx, &ctx->scratch_b, (size_t)ctx->max_cells));
        CKA(dalloc(ctx, &ctx->d_plain_obs, (size_t)ctx->n_traj * ctx->max_nz * 4));
        CKA(dalloc(ctx, &ctx->d_plain_axial, (size_t)ctx->n_traj * ctx->max_nz * 4));
    } else {
        std::vector<GroupParamsF> gfs(ng);
        for (int g = 0; g < ng; ++g) gfs[g] = ctx->groups[g].gf;
        CKA(dalloc(ctx, &ctx->d_gparams, (size_t)ng));
        CKA(cudaMemcpyAsync(ctx->d_gparams, gfs.data(), sizeof(GroupParamsF) * ng, cudaMemcpyHostToDevice, ctx->stream));
        CKA(dalloc(ctx, &ctx->d_step, (size_t)1));
        CKA(dalloc(ctx, &ctx->d_pflags, (size_t)4));
        CKA(cudaMemsetAsync(ctx->d_pflags, 0, 4 * sizeof(int), ctx->stream));
        {
            const char *g = std::getenv("BEC_CUDA_GRAPHS");
            ctx->use_graphs = !(g && g[0] == '0');
        }
        for (auto &c : ctx->classes) {
            const size_t nt = (size_t)c.geom.n_traj;
            c.tiles = fp32_zpass_tiles(c.geom);
            CKA(dalloc(ctx, &c.state, nt * c.geom.cells));
            CKA(cudaMemsetAsync(c.state, 0, sizeof(float4) * nt * c.geom.cells, ctx->stream));
            CKA(dalloc(ctx, &c.d_tgroup, nt));
            CKA(dalloc(ctx, &c.d_tlocal, nt));
            CKA(dalloc(ctx, &c.d_traj_scale, nt));
            const int obs_cap = std::max(c.tiles, fp32_fast_pencil_supported(c.geom) ? fp32_fast_pencil_tiles(c.geom) : 1);
            CKA(dalloc(ctx, &c.obs_partial, nt * obs_cap * c.geom.nz * 4));
            CKA(dalloc(ctx, &c.traj_axial, nt * c.geom.nz * 4));
            std::vector<int> tg(nt), tl(nt);
            std::vector<double> ts(nt);
            for (int g : c.groups) {
                const GroupRec &gr = ctx->groups[g];
                for (int t = 0; t < gr.p.ne; ++t) {
                    tg[gr.local_first + t] = g;
                    tl[gr.local_first + t] = t;
                    ts[gr.local_first + t] = (double)c.geom.nx * c.geom.ny * gr.d.dV;
                }
            }
            CKA(cudaMemcpyAsync(c.d_tgroup, tg.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, ctx->stream));
            CKA(cudaMemcpyAsync(c.d_tlocal, tl.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, ctx->stream));
            CKA(cudaMemcpyAsync(c.d_traj_scale, ts.data(), sizeof(double) * nt, cudaMemcpyHostToDevice, ctx->stream));
            if (fp32_fast_pencil_supported(c.geom)) {
                for (int k = 0; k < 2; ++k) {
                    CKA(dalloc(ctx, &c.kin_tab[k], nt * (size_t)(c.geom.nz + c.geom.nx * c.geom.ny)));
                    fp32_kin_tables(c.kin_tab[k], c.geom, ctx->d_gparams, c.d_tgroup, k ? 1.0f : 0.5f, ctx->stream);
                }
                if (cudaGetLastError() != cudaSuccess) return bail(BEC_ERR_CUDA);
            }
        }
        CKA(dalloc(ctx, &ctx->scratch4, (size_t)ctx->max_cells));
    }
#undef CKA
    (void)st;
    *out = ctx;
    return BEC_OK;
}

void bec_destroy(bec_ctx *ctx)
{
    if (!ctx) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (void *p : ctx->allocs) cudaFree(p);
    step_plan_free(ctx->plan);
    for (auto &t : ctx->ws_tables) cudaFree(t.d_basis);
    for (auto &g : ctx->step_graph)
        if (g) cudaGraphExecDestroy(g);
    for (auto &gr : ctx->groups)
        if (gr.gs_dev) { /* owned through allocs */ }
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev_h2d) cudaEventDestroy(ctx->ev_h2d);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *bec_last_error(const bec_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

bec_status bec_group_info(const bec_ctx *ctx, int32_t group, bec_derived *out)
{
    if (!ctx || !out || group < 0 || group >= (int)ctx->groups.size()) return BEC_ERR_INVALID_ARG;
    *out = ctx->groups[group].d;
    return BEC_OK;
}

int64_t bec_total_trajectories(const bec_ctx *ctx) { return ctx ? ctx->n_traj : 0; }

// ------------------------------------------------------------------------ ground state
bec_status bec_ground_state(bec_ctx *ctx, int32_t group, const bec_gs_opts *opts, double *psi_out,
                            bec_gs_report *rep)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (!opts || !psi_out || group < 0 || group >= (int)ctx->groups.size())
        return fail(ctx, BEC_ERR_INVALID_ARG, "bad ground-state arguments");
    if (opts->mode < BEC_GS_FIXED_STEPS || opts->mode > BEC_GS_MU_RESIDUAL)
        return fail(ctx, BEC_ERR_INVALID_ARG, "unknown ground-state mode");
    GroupRec &gr = ctx->groups[group];
    const GeomD &g = gr.gd;
    const int cells = g.cells;
    cudaStream_t s = ctx->stream;
    const long long l0 = g_launches;
    const bool mu_rule = opts->mode == BEC_GS_MU || opts->mode == BEC_GS_MU_RESIDUAL;
    double2 *a = nullptr, *tmp = nullptr, *tmp2 = nullptr, *prev = nullptr;
    {
        void *pa = nullptr, *pt = nullptr, *pt2 = nullptr, *pp = nullptr;
        CKC(cudaMalloc(&pa, sizeof(double2) * cells));
        if (cudaMalloc(&pt, sizeof(double2) * cells) != cudaSuccess ||
            cudaMalloc(&pt2, sizeof(double2) * cells) != cudaSuccess ||
            (mu_rule && cudaMalloc(&pp, sizeof(double2) * cells) != cudaSuccess)) {
            cudaFree(pa); cudaFree(pt); cudaFree(pt2);
            return fail(ctx, BEC_ERR_OUT_OF_MEMORY, "ground-state buffers");
        }
        a = (double2 *)pa; tmp = (double2 *)pt; tmp2 = (double2 *)pt2; prev = (double2 *)pp;
    }
    struct Guard { void *p[4]; ~Guard() { for (void *q : p) cudaFree(q); } } guard{{a, tmp, tmp2, prev}};
    double *sc = ctx->d_scal;
    double *red = ctx->d_red;
    bec_status st;

    CKC(cudaEventRecord(ctx->ev0, s));
    if (prev) CKC(cudaMemsetAsync(prev, 0, sizeof(double2) * cells, s));
    if (opts->warm_start) {
        CKC(cudaMemcpyAsync(a, opts->warm_start, sizeof(double2) * cells, cudaMemcpyHostToDevice, s));
    } else {
        plain_gs_tf(a, g, gr.d.mu, s);                                  // wigner.cu:97
    }
    plain_norm(a, cells, sc, red, s);                                   // :101-103
    plain_renorm(a, cells, sc, gr.d.N, g.dV, s);
    if ((st = plain_fft(ctx, a, g, 1))) return st;                      // :106-107
    plain_scale(a, cells, 1.0 / cells, s);
    CKL();

    const int maxs = opts->max_steps > 0 ? opts->max_steps : 1;
    const int check = opts->check_every > 0 ? opts->check_every : 1;
    double E = 0.0, mu_prev = 0.0, step_res = 0.0;
    int steps = 0, converged = 0, checks = 0;
    const double res_tol = opts->res_tol > 0.0 ? opts->res_tol : 10.0 * opts->tol;
    auto measure_mu = [&](double *mu_out, double *diff) -> bec_status {
        // x-space sums of the renormalised state, its change since the last check, the Parseval kinetic sum
        plain_gs_xsums(a, g, sc + 8, red, s);
        plain_diff2(a, prev, cells, sc + 20, red, s);
        CKC(cudaMemcpyAsync(prev, a, sizeof(double2) * cells, cudaMemcpyDeviceToDevice, s));
        CKC(cudaMemcpyAsync(tmp, a, sizeof(double2) * cells, cudaMemcpyDeviceToDevice, s));
        bec_status st2 = plain_fft(ctx, tmp, g, 1);
        if (st2) return st2;
        plain_scale(tmp, cells, 1.0 / cells, s);
        plain_gs_ksum(tmp, g, sc + 12, red, s);
        double h[14];
        CKC(cudaMemcpyAsync(h, sc + 8, sizeof(double) * 14, cudaMemcpyDeviceToHost, s));
        CKC(cudaStreamSynchronize(s));
        const double ekin = h[4] * cells * g.dV, epot = h[0] * g.dV, eint = g.g11 * h[1] * g.dV, N = h[2] * g.dV;
        *mu_out = (ekin + epot + eint) / N;
        *diff = std::sqrt(h[12] / h[13]);
        return BEC_OK;
    };
    while (steps < maxs) {
        plain_gs_kick(a, g, s);                                         // :117
        if ((st = plain_fft(ctx, a, g, 0))) return st;                  // :121
        plain_gs_nl(a, g, s);                                           // :124
        if ((st = plain_fft(ctx, a, g, 1))) return st;                  // :129-130
        plain_scale(a, cells, 1.0 / cells, s);
        plain_gs_kick(a, g, s);                                         // :134
        if ((st = plain_fft(ctx, a, g, 0))) return st;                  // :140
        plain_norm(a, cells, sc, red, s);                               // :143-145
        plain_renorm(a, cells, sc, gr.d.N, g.dV, s);
        CKL();
        ++steps;
        bool stop = false;
        if (opts->mode == BEC_GS_REFERENCE_E) {
            CKC(cudaMemcpyAsync(tmp, a, sizeof(double2) * cells, cudaMemcpyDeviceToDevice, s));
            if ((st = plain_fft(ctx, tmp, g, 1))) return st;
            plain_scale(tmp, cells, 1.0 / cells, s);
            plain_gs_ref_energy(a, tmp, g, sc + 1, red, s);
            double hE;
            CKC(cudaMemcpyAsync(&hE, sc + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
            CKC(cudaStreamSynchronize(s));
            const double newE = hE * g.dV;
            if (std::fabs((newE - E) / newE) < 0.000001) stop = true;   // :155
            E = newE;
        } else if (mu_rule && (steps % check) == 0) {
            double mu, diff;
            if ((st = measure_mu(&mu, &diff))) return st;
            if (!std::isfinite(mu)) return fail(ctx, BEC_ERR_NUMERICAL, "ground state diverged");
            const double r = diff / ((double)check * gr.d.dt_steady * std::fabs(mu));
            if (checks > 0) step_res = r;
            const bool mu_ok = mu_prev != 0.0 && std::fabs((mu - mu_prev) / mu) < opts->tol;
            if (mu_ok && (opts->mode == BEC_GS_MU || (checks > 0 && r < res_tol))) stop = true;
            mu_prev = mu;
            ++checks;
        }
        if ((st = plain_fft(ctx, a, g, 1))) return st;                  // :151-152
        plain_scale(a, cells, 1.0 / cells, s);
        if (stop) { converged = 1; break; }
    }
    if ((st = plain_fft(ctx, a, g, 0))) return st;                      // :163
    CKC(cudaEventRecord(ctx->ev1, s));
    CKC(cudaMemcpyAsync(psi_out, a, sizeof(double2) * cells, cudaMemcpyDeviceToHost, s));
    CKC(cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    if (rep) {
        std::memset(rep, 0, sizeof(*rep));
        rep->steps = steps;
        rep->converged = converged;
        rep->seconds = ms * 1e-3;
        rep->step_residual = step_res;
        // mu, energy, residual of the final state
        plain_gs_xsums(a, g, sc + 8, red, s);
        CKC(cudaMemcpyAsync(tmp, a, sizeof(double2) * cells, cudaMemcpyDeviceToDevice, s));
        if ((st = plain_fft(ctx, tmp, g, 1))) return st;
        plain_scale(tmp, cells, 1.0 / cells, s);
        plain_gs_ksum(tmp, g, sc + 12, red, s);
        double h[8];
        CKC(cudaMemcpyAsync(h, sc + 8, sizeof(double) * 8, cudaMemcpyDeviceToHost, s));
        CKC(cudaStreamSynchronize(s));
        const double ekin = h[4] * cells * g.dV, epot = h[0] * g.dV, eint = g.g11 * h[1] * g.dV, N = h[2] * g.dV;
        const double mu = (ekin + epot + eint) / N;
        rep->mu = mu;
        rep->energy = (ekin + epot + 0.5 * eint) / N;
        rep->N = N;
        plain_mul_k2(tmp, tmp2, g, s);
        if ((st = plain_fft(ctx, tmp2, g, 0))) return st;
        plain_gs_residual(a, tmp2, g, mu, sc + 16, red, s);
        double r2;
        CKC(cudaMemcpyAsync(&r2, sc + 16, sizeof(double), cudaMemcpyDeviceToHost, s));
        CKC(cudaStreamSynchronize(s));
        rep->residual = std::sqrt(r2 / h[2]);
    }
    CKL();
    ctx->last_launches = g_launches - l0;
    return BEC_OK;
}

namespace {

// mu, energy per particle, norm and residual of an x-space state already on the device (FP64 kernels)
bec_status plain_measures(bec_ctx *ctx, const GeomD &g, double2 *a, double2 *tmp, double2 *tmp2, bec_gs_report *rep)
{
    cudaStream_t s = ctx->stream;
    double *sc = ctx->d_scal, *red = ctx->d_red;
    const int cells = g.cells;
    bec_status st;
    plain_gs_xsums(a, g, sc + 8, red, s);
    CKC(cudaMemcpyAsync(tmp, a, sizeof(double2) * cells, cudaMemcpyDeviceToDevice, s));
    if ((st = plain_fft(ctx, tmp, g, 1))) return st;
    plain_scale(tmp, cells, 1.0 / cells, s);
    plain_gs_ksum(tmp, g, sc + 12, red, s);
    double h[8];
    CKC(cudaMemcpyAsync(h, sc + 8, sizeof(double) * 8, cudaMemcpyDeviceToHost, s));
    CKC(cudaStreamSynchronize(s));
    const double ekin = h[4] * cells * g.dV, epot = h[0] * g.dV, eint = g.g11 * h[1] * g.dV, N = h[2] * g.dV;
    const double mu = (ekin + epot + eint) / N;
    rep->mu = mu;
    rep->energy = (ekin + epot + 0.5 * eint) / N;
    rep->N = N;
    plain_mul_k2(tmp, tmp2, g, s);
    if ((st = plain_fft(ctx, tmp2, g, 0))) return st;
    plain_gs_residual(a, tmp2, g, mu, sc + 16, red, s);
    double r2;
    CKC(cudaMemcpyAsync(&r2, sc + 16, sizeof(double), cudaMemcpyDeviceToHost, s));
    CKC(cudaStreamSynchronize(s));
    rep->residual = std::sqrt(r2 / h[2]);
    CKL();
    return BEC_OK;
}

struct GsClass {
    ClassGeom geom{};
    std::vector<int> groups;           // group of each local trajectory
    std::vector<int> batch;            // its index in the caller's list
    float2 *state = nullptr, *out = nullptr, *warm = nullptr;
    int *d_tgroup = nullptr;
    int *d_active = nullptr;           // class-local trajectories still iterating (device copy of active)
    std::vector<int> active;
    double *norm = nullptr;            // [2][n]
    double *ekin = nullptr, *xsums = nullptr;
};

// Batched FP32 imaginary-time ground states for groups whose grids the register passes support.
// psi_out (host states) may be NULL; coef_in (n x 64, host) seeds warm starts synthesised on the
// device; coef_out (n x 64, host) receives the projections of the results on the correction basis.
const WsTable *ws_table(const bec_ctx *ctx, int nx, int ny, int nz)
{
    for (const auto &t : ctx->ws_tables)
        if (t.nx == nx && t.ny == ny && t.nz == nz) return &t;
    return nullptr;
}

bec_status gs_batched(bec_ctx *ctx, int n, const int32_t *groups, const bec_gs_opts *opts, double *const *psi_out,
                      bec_gs_report *reports, const double *coef_in = nullptr, double *coef_out = nullptr,
                      float *profile_out = nullptr)
{
    cudaStream_t s = ctx->stream;
    const long long l0 = g_launches;
    std::vector<GsClass> cls;
    std::vector<int> cls_of(n), idx_in(n);
    for (int i = 0; i < n; ++i) {
        const bec_derived &d = ctx->groups[groups[i]].d;
        int c = -1;
        for (size_t k = 0; k < cls.size(); ++k)
            if (cls[k].geom.nx == d.nvx && cls[k].geom.ny == d.nvy && cls[k].geom.nz == d.nvz) c = (int)k;
        if (c < 0) {
            GsClass gc;
            gc.geom.nx = d.nvx; gc.geom.ny = d.nvy; gc.geom.nz = d.nvz;
            gc.geom.lx = ilog2(d.nvx); gc.geom.ly = ilog2(d.nvy); gc.geom.lz = ilog2(d.nvz);
            gc.geom.cells = d.cells;
            cls.push_back(gc);
            c = (int)cls.size() - 1;
        }
        cls_of[i] = c;
        idx_in[i] = (int)cls[c].groups.size();
        cls[c].groups.push_back(groups[i]);
        cls[c].batch.push_back(i);
    }
    // offsets of per-group warm starts (back to back, in list order)
    std::vector<size_t> warm_off(n + 1, 0);
    for (int i = 0; i < n; ++i) warm_off[i + 1] = warm_off[i] + (size_t)ctx->groups[groups[i]].d.cells;
    // per-group FP32 parameters for the whole context (indexed by group)
    std::vector<GsParamsF> hp(ctx->groups.size());
    for (size_t g = 0; g < ctx->groups.size(); ++g) {
        const bec_derived &d = ctx->groups[g].d;
        hp[g].N = d.N;
        hp[g].parseval = (double)d.cells * d.dV;
        hp[g].dt_steady = (float)d.dt_steady;
        hp[g].mu = (float)d.mu;
    }
    std::vector<void *> tmp_allocs;
    struct Free { std::vector<void *> &v; cudaStream_t s; ~Free() { cudaStreamSynchronize(s); for (void *p : v) cudaFree(p); } } fr{tmp_allocs, s};
    auto talloc = [&](void **p, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaMalloc(p, bytes > 0 ? bytes : 16);
        if (e == cudaSuccess) tmp_allocs.push_back(*p);
        return e;
    };
    GsParamsF *d_gs = nullptr;
    CKC(talloc((void **)&d_gs, sizeof(GsParamsF) * hp.size()));
    CKC(cudaMemcpyAsync(d_gs, hp.data(), sizeof(GsParamsF) * hp.size(), cudaMemcpyHostToDevice, s));
    // GroupParamsF of every group (the batched context has them already; the plain one does not)
    GroupParamsF *d_gp = ctx->d_gparams;
    if (!d_gp) {
        std::vector<GroupParamsF> gfs(ctx->groups.size());
        for (size_t g = 0; g < gfs.size(); ++g) gfs[g] = ctx->groups[g].gf;
        CKC(talloc((void **)&d_gp, sizeof(GroupParamsF) * gfs.size()));
        CKC(cudaMemcpyAsync(d_gp, gfs.data(), sizeof(GroupParamsF) * gfs.size(), cudaMemcpyHostToDevice, s));
    }
    // allocations and host-side staging first: the timed region holds the device work from the first copy on
    // (cudaMalloc of fresh memory can hold the host for tens of ms, which the device clock would count)
    std::vector<std::vector<float2>> warm_h(cls.size());
    std::vector<std::vector<double>> warm_cc(cls.size());
    std::vector<std::vector<bec_derived>> warm_dd(cls.size());
    for (size_t k = 0; k < cls.size(); ++k) {
        GsClass &c = cls[k];
        const size_t nt = c.groups.size(), cells = c.geom.cells;
        c.geom.n_traj = (int)nt;
        CKC(talloc((void **)&c.state, sizeof(float2) * nt * cells));
        CKC(talloc((void **)&c.out, sizeof(float2) * nt * cells));
        CKC(talloc((void **)&c.d_tgroup, sizeof(int) * nt));
        CKC(talloc((void **)&c.d_active, sizeof(int) * nt));
        CKC(talloc((void **)&c.norm, sizeof(double) * 2 * nt));
        CKC(talloc((void **)&c.ekin, sizeof(double) * nt));
        CKC(talloc((void **)&c.xsums, sizeof(double) * 4 * nt));
        c.active.resize(nt);
        for (size_t t = 0; t < nt; ++t) c.active[t] = (int)t;
        if (opts->warm_start) {
            std::vector<float2> &h = warm_h[k];
            h.resize(nt * cells);
            for (size_t t = 0; t < nt; ++t)
                for (size_t i = 0; i < cells; ++i) {
                    const size_t src = (opts->warm_per_group ? warm_off[c.batch[t]] : 0) + i;
                    h[t * cells + i] = make_float2((float)opts->warm_start[2 * src], (float)opts->warm_start[2 * src + 1]);
                }
            CKC(talloc((void **)&c.warm, sizeof(float2) * nt * cells));
        } else if (coef_in) {
            const int nb = warmstart_basis_size();
            std::vector<double> &cc = warm_cc[k];
            std::vector<bec_derived> &dd = warm_dd[k];
            cc.resize(nt * nb);
            dd.resize(nt);
            for (size_t t = 0; t < nt; ++t) {
                dd[t] = ctx->groups[c.groups[t]].d;
                for (int k2 = 0; k2 < nb; ++k2) cc[t * nb + k2] = coef_in[(size_t)c.batch[t] * nb + k2];
            }
            CKC(talloc((void **)&c.warm, sizeof(float2) * nt * cells));
        }
    }
    CKC(cudaEventRecord(ctx->ev0, s));      // the timed region includes the warm-start synthesis
    for (size_t k = 0; k < cls.size(); ++k) {
        GsClass &c = cls[k];
        const size_t nt = c.groups.size(), cells = c.geom.cells;
        CKC(cudaMemcpyAsync(c.d_active, c.active.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, s));
        CKC(cudaMemsetAsync(c.out, 0, sizeof(float2) * nt * cells, s));   // the first check sees a full change
        CKC(cudaMemcpyAsync(c.d_tgroup, c.groups.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, s));
        CKC(cudaMemsetAsync(c.norm, 0, sizeof(double) * 2 * nt, s));
        if (opts->warm_start)
            CKC(cudaMemcpyAsync(c.warm, warm_h[k].data(), sizeof(float2) * warm_h[k].size(), cudaMemcpyHostToDevice, s));
        else if (coef_in)
            CKC(warmstart_synth(warm_cc[k].data(), (int)nt, warm_dd[k].data(),
                                ws_table(ctx, c.geom.nx, c.geom.ny, c.geom.nz), c.warm, s));
    }
    auto tw_for = [&](int nz, float2 **tw) { return get_tw32_full_nearest(ctx, nz, tw); };
    bec_status st;
    // start: x-space profile -> stored form; measure its norm, first half kick of step 0
    for (auto &c : cls) {
        float2 *tw;
        if ((st = tw_for(c.geom.nz, &tw))) return st;
        gs_init(c.state, c.geom, d_gp, d_gs, c.d_tgroup, c.warm, s);
        gs_prep(c.state, c.geom, d_gp, d_gs, c.d_tgroup, s);
        gs_pencil(c.state, c.geom, d_gp, d_gs, c.d_tgroup, tw, 0.0f, 0.5f, 1.0f / c.geom.cells, 1.0f, c.norm,
                  nullptr, s);
    }
    CKL();
    const int maxs = opts->max_steps > 0 ? opts->max_steps : 1;
    const int check = opts->check_every > 0 ? opts->check_every : 1;
    const bool mu_mode = opts->mode == BEC_GS_MU || opts->mode == BEC_GS_MU_RESIDUAL;
    const double res_tol = opts->res_tol > 0.0 ? opts->res_tol : 10.0 * opts->tol;
    std::vector<std::vector<double>> mu_prev(cls.size()), conv_step(cls.size()), step_res(cls.size());
    for (size_t k = 0; k < cls.size(); ++k) {
        mu_prev[k].assign(cls[k].groups.size(), 0.0);
        conv_step[k].assign(cls[k].groups.size(), -1.0);
        step_res[k].assign(cls[k].groups.size(), 0.0);
    }
    int steps = 0, checks = 0;
    bool converged_all = false;
    // measures the boundary state after `steps` steps: writes out (renormalised x-space), mu per trajectory
    // and the relative change of the state since the previous boundary
    // launches cover the active trajectories only; per-trajectory buffers stay indexed by class-local position
    auto run_geom = [](const GsClass &c) { ClassGeom g = c.geom; g.n_traj = (int)c.active.size(); return g; };
    auto boundary = [&](bool final_pass, std::vector<std::vector<double>> *mus,
                        std::vector<std::vector<double>> *diffs) -> bec_status {
        const int b = steps & 1;            // buffer the closing pencil pass measures into
        for (auto &c : cls) {
            if (c.active.empty()) continue;
            float2 *tw;
            bec_status st2;
            if ((st2 = tw_for(c.geom.nz, &tw))) return st2;
            const int nt = c.geom.n_traj;
            const ClassGeom ag = run_geom(c);
            CKC(cudaMemsetAsync(c.ekin, 0, sizeof(double) * nt, s));
            CKC(cudaMemsetAsync(c.xsums, 0, sizeof(double) * 4 * nt, s));
            gs_pencil(c.state, ag, d_gp, d_gs, c.d_tgroup, tw, 0.5f, 0.0f, 1.0f / c.geom.cells,
                      (float)(c.geom.nx * c.geom.ny), c.norm + (size_t)b * nt, c.ekin, s, c.d_active);
            gs_output(c.state, ag, d_gp, d_gs, c.d_tgroup, c.norm + (size_t)b * nt, c.out, c.xsums,
                      1.0f / (float)(c.geom.nx * c.geom.ny), s, c.d_active);
            if (!final_pass)   // resume: first half kick of the next step, norm already measured
                gs_pencil(c.state, ag, d_gp, d_gs, c.d_tgroup, tw, 0.0f, 0.5f, 1.0f / c.geom.cells, 1.0f,
                          nullptr, nullptr, s, c.d_active);
        }
        CKL();
        if (mus) {
            for (size_t k = 0; k < cls.size(); ++k) {
                auto &c = cls[k];
                const int nt = c.geom.n_traj;
                std::vector<double> nrm(nt), ek(nt), xs(4 * nt);
                CKC(cudaMemcpyAsync(nrm.data(), c.norm + (size_t)b * nt, sizeof(double) * nt, cudaMemcpyDeviceToHost, s));
                CKC(cudaMemcpyAsync(ek.data(), c.ekin, sizeof(double) * nt, cudaMemcpyDeviceToHost, s));
                CKC(cudaMemcpyAsync(xs.data(), c.xsums, sizeof(double) * 4 * nt, cudaMemcpyDeviceToHost, s));
                CKC(cudaStreamSynchronize(s));
                (*mus)[k].assign(nt, 0.0);
                (*diffs)[k].assign(nt, 0.0);
                for (int t : c.active) {
                    const bec_derived &d = ctx->groups[c.groups[t]].d;
                    const double s2 = d.N / (nrm[t] * (double)d.cells * d.dV);       // renormalisation squared
                    const double e_kin = ek[t] * s2 * (double)d.cells * d.dV;
                    const double N = xs[4 * t + 2] * d.dV;
                    (*mus)[k][t] = (e_kin + xs[4 * t] * d.dV + d.g11 * xs[4 * t + 1] * d.dV) / N;
                    (*diffs)[k][t] = std::sqrt(xs[4 * t + 3] / xs[4 * t + 2]);
                }
            }
        }
        return BEC_OK;
    };
    while (steps < maxs) {
        const int b = steps & 1;
        for (auto &c : cls) {
            if (c.active.empty()) continue;
            const int nt = c.geom.n_traj;
            gs_plane_step(c.state, run_geom(c), d_gp, d_gs, c.d_tgroup, c.norm + (size_t)b * nt,
                          c.norm + (size_t)(b ^ 1) * nt, s, c.d_active);
        }
        CKL();
        ++steps;
        const bool last = steps == maxs;
        if (mu_mode && (steps % check) == 0 && !last) {
            std::vector<std::vector<double>> mus(cls.size()), diffs(cls.size());
            if ((st = boundary(false, &mus, &diffs))) return st;
            bool all = true;
            for (size_t k = 0; k < cls.size(); ++k) {
                for (int t : cls[k].active) {
                    const double m = mus[k][t];
                    if (!std::isfinite(m)) return fail(ctx, BEC_ERR_NUMERICAL, "ground state diverged");
                    const double dt = ctx->groups[cls[k].groups[t]].d.dt_steady;
                    const double r = diffs[k][t] / ((double)check * dt * std::fabs(m));
                    if (checks > 0) step_res[k][t] = r;
                    const bool mu_ok = mu_prev[k][t] != 0.0 && std::fabs((m - mu_prev[k][t]) / m) < opts->tol;
                    if (conv_step[k][t] < 0 && mu_ok &&
                        (opts->mode == BEC_GS_MU || (checks > 0 && r < res_tol)))
                        conv_step[k][t] = steps;
                    mu_prev[k][t] = m;
                }
                // converged trajectories leave the batch; their out keeps the state they converged in
                std::vector<int> still;
                for (int t : cls[k].active)
                    if (conv_step[k][t] < 0) still.push_back(t);
                if (still.size() != cls[k].active.size()) {
                    cls[k].active = still;
                    if (!still.empty())
                        CKC(cudaMemcpyAsync(cls[k].d_active, still.data(), sizeof(int) * still.size(),
                                            cudaMemcpyHostToDevice, s));
                }
                all = all && cls[k].active.empty();
            }
            ++checks;
            if (all) { converged_all = true; break; }
        } else if (!last) {
            for (auto &c : cls) {
                if (c.active.empty()) continue;
                float2 *tw;
                if ((st = tw_for(c.geom.nz, &tw))) return st;
                const int nt = c.geom.n_traj;
                gs_pencil(c.state, run_geom(c), d_gp, d_gs, c.d_tgroup, tw, 0.5f, 0.5f, 1.0f / c.geom.cells, 1.0f,
                          c.norm + (size_t)((steps & 1)) * nt, nullptr, s, c.d_active);
            }
            CKL();
        }
    }
    // trajectories that converged at a check already hold their renormalised state in out
    if (!converged_all && (st = boundary(true, nullptr, nullptr))) return st;
    CKC(cudaEventRecord(ctx->ev1, s));
    CKC(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    // outputs, FP64 measures of each ground state on the device
    size_t maxc = 0;
    for (auto &c : cls) maxc = std::max(maxc, (size_t)c.geom.cells);
    double2 *a64 = nullptr, *t1 = nullptr, *t2 = nullptr;
    CKC(talloc((void **)&a64, sizeof(double2) * maxc));
    CKC(talloc((void **)&t1, sizeof(double2) * maxc));
    CKC(talloc((void **)&t2, sizeof(double2) * maxc));
    for (int i = 0; i < n; ++i) {
        GsClass &c = cls[cls_of[i]];
        const size_t cells = c.geom.cells;
        const float2 *src = c.out + (size_t)idx_in[i] * cells;
        if (psi_out) {
            std::vector<float2> h(cells);
            CKC(cudaMemcpyAsync(h.data(), src, sizeof(float2) * cells, cudaMemcpyDeviceToHost, s));
            CKC(cudaStreamSynchronize(s));
            for (size_t k = 0; k < cells; ++k) { psi_out[i][2 * k] = h[k].x; psi_out[i][2 * k + 1] = h[k].y; }
        }
        if (reports) {
            bec_gs_report &r = reports[i];
            std::memset(&r, 0, sizeof(r));
            const double cs = conv_step[cls_of[i]][idx_in[i]];
            r.converged = mu_mode ? (cs >= 0 ? 1 : 0) : 0;
            r.steps = (mu_mode && cs >= 0) ? (int)cs : steps;
            r.step_residual = step_res[cls_of[i]][idx_in[i]];
            r.seconds = ms * 1e-3;
            gs_to_double(src, a64, cells, s);
            if ((st = plain_measures(ctx, ctx->groups[groups[i]].gd, a64, t1, t2, &r))) return st;
        }
    }
    if (coef_out || profile_out) {
        const int nb = warmstart_basis_size();
        for (auto &c : cls) {
            const size_t nt = c.groups.size(), cells = c.geom.cells;
            std::vector<bec_derived> dd(nt);
            for (size_t t = 0; t < nt; ++t) dd[t] = ctx->groups[c.groups[t]].d;
            std::vector<double> cc(nt * nb);
            std::vector<float> pr(profile_out ? nt * cells : 0);
            CKC(warmstart_project(c.out, (int)nt, dd.data(), ws_table(ctx, c.geom.nx, c.geom.ny, c.geom.nz),
                                  coef_out ? cc.data() : nullptr, profile_out ? pr.data() : nullptr, s));
            for (size_t t = 0; t < nt; ++t) {
                if (coef_out)
                    for (int k = 0; k < nb; ++k) coef_out[(size_t)c.batch[t] * nb + k] = cc[t * nb + k];
                if (profile_out)
                    std::memcpy(profile_out + (size_t)c.batch[t] * cells, pr.data() + t * cells, sizeof(float) * cells);
            }
        }
    }
    ctx->last_launches = g_launches - l0;
    ctx->last_ms = ms;
    return BEC_OK;
}

} // namespace

bec_status bec_ground_state_coeffs(bec_ctx *ctx, int32_t n, const int32_t *groups, const bec_gs_opts *opts,
                                   const double *coef_in, double *coef_out, float *profile_out,
                                   bec_gs_report *reports)
{
    if (!ctx || n < 1 || !groups || !opts) return BEC_ERR_INVALID_ARG;
    if (opts->mode < BEC_GS_FIXED_STEPS || opts->mode > BEC_GS_MU_RESIDUAL)
        return fail(ctx, BEC_ERR_INVALID_ARG, "unknown ground-state mode");
    if (ctx->path != BEC_PATH_FP32_BATCHED || opts->mode == BEC_GS_REFERENCE_E || opts->warm_start)
        return fail(ctx, BEC_ERR_INVALID_ARG, "coefficient ground states need the batched path and a FIXED or MU rule");
    const bec_derived &d0 = ctx->groups[groups[0]].d;
    for (int i = 0; i < n; ++i) {
        if (groups[i] < 0 || groups[i] >= (int)ctx->groups.size()) return fail(ctx, BEC_ERR_INVALID_ARG, "bad group");
        const bec_derived &d = ctx->groups[groups[i]].d;
        ClassGeom g{};
        g.nx = d.nvx; g.ny = d.nvy; g.nz = d.nvz; g.n_traj = 4;
        if (d.nvx != d0.nvx || d.nvy != d0.nvy || d.nvz != d0.nvz || !gs_batched_supported(g))
            return fail(ctx, BEC_ERR_UNSUPPORTED_GRID, "coefficient ground states need one supported grid");
    }
    return gs_batched(ctx, n, groups, opts, nullptr, reports, coef_in, coef_out, profile_out);
}

int32_t bec_warmstart_basis_size(void) { return warmstart_basis_size(); }

bec_status bec_warmstart_set_basis(bec_ctx *ctx, int32_t nvx, int32_t nvy, int32_t nvz, int32_t nb,
                                   const float *basis)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (nvx < 2 || nvy < 1 || nvz < 2 || (nvx & (nvx - 1)) || (nvy & (nvy - 1)) || (nvz & (nvz - 1)) || nb < 0 ||
        nb > warmstart_basis_size() || (nb > 0 && !basis))
        return fail(ctx, BEC_ERR_INVALID_ARG, "bad warm-start basis arguments");
    for (size_t i = 0; i < ctx->ws_tables.size(); ++i) {
        WsTable &t = ctx->ws_tables[i];
        if (t.nx == nvx && t.ny == nvy && t.nz == nvz) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(t.d_basis);
            ctx->ws_tables.erase(ctx->ws_tables.begin() + i);
            break;
        }
    }
    if (nb == 0 || !basis) return BEC_OK;
    WsTable t;
    t.nx = nvx; t.ny = nvy; t.nz = nvz; t.nb = nb;
    const cudaError_t e = warmstart_table_init(t, basis, ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(t.d_basis);
        if (e == cudaErrorInvalidValue) return fail(ctx, BEC_ERR_INVALID_ARG, "warm-start basis rows are dependent");
        return fail(ctx, e == cudaErrorMemoryAllocation ? BEC_ERR_OUT_OF_MEMORY : BEC_ERR_CUDA,
                    std::string("warm-start basis: ") + cudaGetErrorString(e));
    }
    ctx->ws_tables.push_back(t);
    return BEC_OK;
}

bec_status bec_ground_state_batch(bec_ctx *ctx, int32_t n, const int32_t *groups, const bec_gs_opts *opts,
                                  double *const *psi_out, bec_gs_report *reports)
{
    if (!ctx || n < 0 || (n > 0 && (!groups || !psi_out || !opts))) return BEC_ERR_INVALID_ARG;
    if (n > 0 && (opts->mode < BEC_GS_FIXED_STEPS || opts->mode > BEC_GS_MU_RESIDUAL))
        return fail(ctx, BEC_ERR_INVALID_ARG, "unknown ground-state mode");
    for (int i = 0; i < n; ++i)
        if (groups[i] < 0 || groups[i] >= (int)ctx->groups.size() || !psi_out[i])
            return fail(ctx, BEC_ERR_INVALID_ARG, "bad group index or output pointer");
    // the batched FP32 path: FIXED_STEPS, MU or MU_RESIDUAL rules on grids the register passes cover
    bool batched = ctx->path == BEC_PATH_FP32_BATCHED && opts->mode != BEC_GS_REFERENCE_E && n > 0;
    for (int i = 0; batched && i < n; ++i) {
        const bec_derived &d = ctx->groups[groups[i]].d;
        ClassGeom g{};
        g.nx = d.nvx; g.ny = d.nvy; g.nz = d.nvz; g.n_traj = 4;
        if (!gs_batched_supported(g)) batched = false;
    }
    if (batched) return gs_batched(ctx, n, groups, opts, psi_out, reports);
    for (int i = 0; i < n; ++i) {
        bec_status st = bec_ground_state(ctx, groups[i], opts, psi_out[i], reports ? &reports[i] : nullptr);
        if (st) return st;
    }
    return BEC_OK;
}

// ------------------------------------------------------------------------ evolution
namespace {
// The staging area of the ground states an init call copies to the device: every group's slot in group
// order, 16 bytes per cell. A ground state is consumed by the call that copies it, so bec_init_group and
// bec_init_groups share the area; whichever runs first allocates it.
bec_status gs_stage_ready(bec_ctx *ctx)
{
    if (ctx->gs_stage) return BEC_OK;
    size_t total = 0;
    for (auto &gr : ctx->groups) total += sizeof(double2) * (size_t)gr.gd.cells;
    CKC(dalloc(ctx, &ctx->gs_stage, total));
    return BEC_OK;
}
} // namespace

bec_status bec_init_group(bec_ctx *ctx, int32_t group, const double *psi_gs, const double *noise)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (!psi_gs || group < 0 || group >= (int)ctx->groups.size())
        return fail(ctx, BEC_ERR_INVALID_ARG, "bad init arguments");
    GroupRec &gr = ctx->groups[group];
    const GeomD &g = gr.gd;
    const int cells = g.cells, ne = gr.p.ne;
    cudaStream_t s = ctx->stream;
    bec_status st;
    const long long l0 = g_launches;
    if (ctx->path == BEC_PATH_FP64_PLAIN) {
        double2 *gs = ctx->scratch_a, *nz = nullptr;
        CKC(cudaMemcpyAsync(gs, psi_gs, sizeof(double2) * cells, cudaMemcpyHostToDevice, s));
        CKC(cudaEventRecord(ctx->ev_h2d, s));
        if (noise) {
            void *p = nullptr;
            CKC(cudaMalloc(&p, sizeof(double2) * 2 * (size_t)cells * ne));
            nz = (double2 *)p;
            cudaError_t e = cudaMemcpyAsync(nz, noise, sizeof(double2) * 2 * (size_t)cells * ne,
                                            cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) { cudaFree(p); return fail(ctx, BEC_ERR_CUDA, cudaGetErrorString(e)); }
        }
        for (int t = 0; t < ne; ++t) {
            double2 *a = gr.a + (size_t)t * cells, *b = gr.b + (size_t)t * cells;
            plain_init(a, b, gs, nz ? nz + (size_t)(2 * t) * cells : nullptr,
                       nz ? nz + (size_t)(2 * t + 1) * cells : nullptr, g, (uint32_t)t, s);
            if ((st = plain_fft(ctx, a, g, 1))) { if (nz) { cudaStreamSynchronize(s); cudaFree(nz); } return st; }
            if ((st = plain_fft(ctx, b, g, 1))) { if (nz) { cudaStreamSynchronize(s); cudaFree(nz); } return st; }
            plain_scale(a, cells, 1.0 / cells, s);
            plain_scale(b, cells, 1.0 / cells, s);
        }
        if (nz) { cudaStreamSynchronize(s); cudaFree(nz); }
        CKL();
    } else {
        // bring the other groups to a clean step boundary first
        if ((st = batched_resolve(ctx, false))) return st;
        if ((st = gs_stage_ready(ctx))) return st;
        size_t off = 0;
        for (int g = 0; g < group; ++g) off += sizeof(double2) * (size_t)ctx->groups[g].gd.cells;
        gr.gs_dev = reinterpret_cast<double2 *>(ctx->gs_stage + off);
        CKC(cudaMemcpyAsync(gr.gs_dev, psi_gs, sizeof(double2) * cells, cudaMemcpyHostToDevice, s));
        CKC(cudaEventRecord(ctx->ev_h2d, s));
        float2 *nz = nullptr;
        if (noise) {
            std::vector<float2> h((size_t)2 * cells * ne);
            for (size_t i = 0; i < h.size(); ++i) h[i] = make_float2((float)noise[2 * i], (float)noise[2 * i + 1]);
            void *p = nullptr;
            CKC(cudaMalloc(&p, sizeof(float2) * h.size()));
            nz = (float2 *)p;
            cudaError_t e = cudaMemcpyAsync(nz, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice, ctx->stream);
            if (e != cudaSuccess) { cudaFree(p); return fail(ctx, BEC_ERR_CUDA, cudaGetErrorString(e)); }
        }
        ClassRec &c = ctx->classes[gr.cls];
        float4 *base = c.state + (size_t)gr.local_first * cells;
        fp32_init_group(base, cells, ne, gr.gf, gr.gs_dev, nz, s);
        ClassGeom sub = c.geom;
        sub.n_traj = ne;
        float2 *tx, *ty;
        if ((st = get_tw32(ctx, sub.nx, &tx)) || (st = get_tw32(ctx, sub.ny, &ty))) {
            if (nz) { cudaStreamSynchronize(s); cudaFree(nz); }
            return st;
        }
        fp32_prep(base, sub, tx, ty, s);
        if (nz) { cudaStreamSynchronize(s); cudaFree(nz); }
        CKL();
    }
    gr.initialised = true;
    ctx->last_launches = g_launches - l0;
    // the caller may reuse psi_gs once this returns: wait for its copy (the kernels behind it keep running)
    CKC(cudaEventSynchronize(ctx->ev_h2d));
    return BEC_OK;
}

bec_status bec_init_groups(bec_ctx *ctx, int32_t n, const int32_t *groups, const void *const *psi_gs,
                           int32_t host_type)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (n < 0 || (n > 0 && (!groups || !psi_gs)) ||
        (host_type != BEC_HOST_C128 && host_type != BEC_HOST_C64 && host_type != BEC_HOST_R32))
        return fail(ctx, BEC_ERR_INVALID_ARG, "bad bec_init_groups arguments");
    const int ng = (int)ctx->groups.size();
    std::vector<char> listed(ng, 0);
    for (int i = 0; i < n; ++i) {
        const int g = groups[i];
        if (g < 0 || g >= ng || listed[g] || !psi_gs[i])
            return fail(ctx, BEC_ERR_INVALID_ARG, "bec_init_groups: group index out of range, repeated or NULL");
        listed[g] = 1;
    }
    const bool c64 = host_type == BEC_HOST_C64;
    bec_status st;
    if (ctx->path == BEC_PATH_FP64_PLAIN) {
        const long long l0 = g_launches;
        for (int i = 0; i < n; ++i) {
            if (c64 || host_type == BEC_HOST_R32) {
                const int cells = ctx->groups[groups[i]].gd.cells;
                const float *f = static_cast<const float *>(psi_gs[i]);
                std::vector<double> d(2 * (size_t)cells, 0.0);
                for (size_t k = 0; k < (size_t)cells; ++k) {
                    if (c64) { d[2 * k] = f[2 * k]; d[2 * k + 1] = f[2 * k + 1]; }
                    else d[2 * k] = f[k];
                }
                if ((st = bec_init_group(ctx, groups[i], d.data(), nullptr))) return st;
            } else if ((st = bec_init_group(ctx, groups[i], static_cast<const double *>(psi_gs[i]), nullptr))) {
                return st;
            }
        }
        ctx->last_launches = g_launches - l0;
        return BEC_OK;
    }
    if ((st = batched_resolve(ctx, false))) return st;
    const long long l0 = g_launches;
    cudaStream_t s = ctx->stream;
    if (!ctx->d_gs_ptrs) CKC(dalloc(ctx, &ctx->d_gs_ptrs, (size_t)ng));
    // the staging area holds the listed ground states in group order at the call's element size, so that
    // consecutive groups whose host buffers are adjacent arrive in one copy
    const size_t esz = host_type == BEC_HOST_R32 ? sizeof(float) : c64 ? sizeof(float2) : sizeof(double2);
    std::vector<size_t> off(ng + 1, 0);
    for (int g = 0; g < ng; ++g) off[g + 1] = off[g] + esz * (size_t)ctx->groups[g].gd.cells;
    if ((st = gs_stage_ready(ctx))) return st;
    for (int i = 0; i < n;) {
        int k = i + 1;
        const char *h0 = static_cast<const char *>(psi_gs[i]);
        while (k < n && groups[k] == groups[k - 1] + 1 &&
               static_cast<const char *>(psi_gs[k]) == h0 + (off[groups[k]] - off[groups[i]]))
            ++k;
        CKC(cudaMemcpyAsync(ctx->gs_stage + off[groups[i]], h0, off[groups[k - 1] + 1] - off[groups[i]],
                            cudaMemcpyHostToDevice, s));
        i = k;
    }
    std::vector<const void *> tab(ng);
    for (int g = 0; g < ng; ++g) tab[g] = ctx->gs_stage + off[g];
    if (tab != ctx->gs_ptrs_host) {
        // pageable source: the copy is staged before the call returns, so tab may go out of scope
        CKC(cudaMemcpyAsync(ctx->d_gs_ptrs, tab.data(), sizeof(void *) * ng, cudaMemcpyHostToDevice, s));
        ctx->gs_ptrs_host = tab;
    }
    CKC(cudaEventRecord(ctx->ev_h2d, s));
    // one initialisation kernel and one preparation pass per run of consecutive listed trajectories
    for (auto &c : ctx->classes) {
        std::vector<std::pair<int, int>> runs;    // (first local trajectory, count)
        std::vector<int> gl;
        for (int g : c.groups)
            if (listed[g]) gl.push_back(g);
        std::sort(gl.begin(), gl.end(), [&](int a, int b) { return ctx->groups[a].local_first < ctx->groups[b].local_first; });
        for (int g : gl) {
            const GroupRec &gr = ctx->groups[g];
            if (!runs.empty() && runs.back().first + runs.back().second == gr.local_first) runs.back().second += gr.p.ne;
            else runs.push_back({gr.local_first, gr.p.ne});
        }
        for (const auto &r : runs) {
            float4 *base = c.state + (size_t)r.first * c.geom.cells;
            fp32_init_batched(base, c.geom.cells, r.second, c.d_tgroup + r.first, c.d_tlocal + r.first, ctx->d_gparams,
                              ctx->d_gs_ptrs, host_type, s);
            CKL();
            ClassGeom sub = c.geom;
            sub.n_traj = r.second;
            float2 *tx, *ty;
            if ((st = get_tw32(ctx, sub.nx, &tx)) || (st = get_tw32(ctx, sub.ny, &ty))) return st;
            fp32_prep(base, sub, tx, ty, s);
            CKL();
        }
    }
    for (int i = 0; i < n; ++i) ctx->groups[groups[i]].initialised = true;
    ctx->last_launches = g_launches - l0;
    // the caller may reuse psi_gs once this returns: wait for the copies (the kernels behind them keep running)
    CKC(cudaEventSynchronize(ctx->ev_h2d));
    return BEC_OK;
}

bec_status bec_evolve(bec_ctx *ctx, int32_t n_steps)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (n_steps < 0) return fail(ctx, BEC_ERR_INVALID_ARG, "negative step count");
    bec_status st = check_ready(ctx);
    if (st) return st;
    // the schedule autotuner times its candidates with the same events; it normally runs in the equilibration
    // step of bec_start_evolution, and never inside this call's timed region
    if ((st = ensure_plan(ctx))) return st;
    const long long l0 = g_launches;
    CKC(cudaEventRecord(ctx->ev0, ctx->stream));
    if ((st = do_evolve(ctx, n_steps))) return st;
    CKC(cudaEventRecord(ctx->ev1, ctx->stream));
    CKC(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->last_ms = ms;
    ctx->last_launches = g_launches - l0;
    return check_step_error(ctx);
}

bec_status bec_pulse(bec_ctx *ctx, double theta, double phi)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    bec_status st = check_ready(ctx);
    if (st) return st;
    double2 m[4];
    rotation(theta, phi, m);
    return apply_pulse(ctx, m);
}

bec_status bec_pulse_finite(bec_ctx *ctx, double rabi_hz, double duration_s, double phi)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (!(duration_s > 0) || !std::isfinite(rabi_hz) || !std::isfinite(phi))
        return fail(ctx, BEC_ERR_INVALID_ARG, "bad pulse parameters");
    bec_status st = check_ready(ctx);
    if (st) return st;
    const double dt = ctx->groups[0].p.dt_evo;
    for (auto &g : ctx->groups)
        if (g.p.dt_evo != dt) return fail(ctx, BEC_ERR_INVALID_ARG, "finite pulses need one dt_evo for all groups");
    const long long n = std::max(1LL, (long long)std::llround(duration_s / dt));
    const double half = 0.5 * 2.0 * M_PI * rabi_hz * (duration_s / (double)n);   // Omega dt_sub / 2
    double2 m[4];
    rotation(half, phi, m);
    const long long l0 = g_launches;
    for (long long k = 0; k < n; ++k) {
        if ((st = apply_pulse(ctx, m))) return st;
        if ((st = do_evolve(ctx, 1))) return st;
        if ((st = apply_pulse(ctx, m))) return st;
    }
    ctx->last_launches = g_launches - l0;
    CKC(cudaStreamSynchronize(ctx->stream));
    return check_step_error(ctx);
}

bec_status bec_start_evolution(bec_ctx *ctx)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    bec_status st = check_ready(ctx);
    if (st) return st;
    int neq = ctx->groups[0].d.n_equil_steps;
    for (auto &g : ctx->groups)
        if (g.d.n_equil_steps != neq)
            return fail(ctx, BEC_ERR_INVALID_ARG, "groups disagree on the equilibration step count");
    if ((st = do_evolve(ctx, neq))) return st;                     // wigner.cu:222-223
    double2 m[4];
    rotation(M_PI / 2.0, 0.0, m);                                   // wigner.cu:225
    if ((st = apply_pulse(ctx, m))) return st;
    ctx->evo_steps = 0;
    CKC(cudaStreamSynchronize(ctx->stream));
    return check_step_error(ctx);
}

bec_status bec_moments_now(bec_ctx *ctx, bec_moments *out)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (!out) return fail(ctx, BEC_ERR_INVALID_ARG, "null output");
    bec_status st = check_ready(ctx);
    if (st) return st;
    if ((st = observe_now(ctx))) return st;
    return fetch_group_moments(ctx, out);
}

bec_status bec_traj_moments_now(bec_ctx *ctx, bec_moments *out)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (!out) return fail(ctx, BEC_ERR_INVALID_ARG, "null output");
    bec_status st = check_ready(ctx);
    if (st) return st;
    if ((st = observe_now(ctx))) return st;
    std::vector<double> h((size_t)ctx->n_traj * 4);
    CKC(cudaMemcpyAsync(h.data(), ctx->d_traj_tot, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ctx->stream));
    CKC(cudaStreamSynchronize(ctx->stream));
    for (auto &gr : ctx->groups)
        for (int t = 0; t < gr.p.ne; ++t) {
            const int i = gr.traj_first + t;
            out[i].t = ctx->evo_steps * gr.p.dt_evo;
            out[i].na = h[i * 4 + 0]; out[i].nb = h[i * 4 + 1];
            out[i].s_re = h[i * 4 + 2]; out[i].s_im = h[i * 4 + 3];
        }
    return BEC_OK;
}

static bec_status group_axial_host(bec_ctx *ctx, int group, double *out)
{
    GroupRec &gr = ctx->groups[group];
    const int nz = gr.d.nvz;
    std::vector<double> h;
    if (ctx->path == BEC_PATH_FP64_PLAIN) {
        h.resize((size_t)gr.p.ne * ctx->max_nz * 4);
        CKC(cudaMemcpyAsync(h.data(), ctx->d_plain_axial + (size_t)gr.traj_first * ctx->max_nz * 4,
                            sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ctx->stream));
    } else {
        ClassRec &c = ctx->classes[gr.cls];
        h.resize((size_t)gr.p.ne * nz * 4);
        CKC(cudaMemcpyAsync(h.data(), c.traj_axial + (size_t)gr.local_first * nz * 4, sizeof(double) * h.size(),
                            cudaMemcpyDeviceToHost, ctx->stream));
    }
    CKC(cudaStreamSynchronize(ctx->stream));
    const int row = (ctx->path == BEC_PATH_FP64_PLAIN) ? ctx->max_nz : nz;
    for (int z = 0; z < nz; ++z)
        for (int k = 0; k < 4; ++k) {
            HSum acc;
            for (int t = 0; t < gr.p.ne; ++t) acc.add(h[((size_t)t * row + z) * 4 + k]);
            out[4 * z + k] = acc.value();
        }
    return BEC_OK;
}

bec_status bec_axial_now(bec_ctx *ctx, int32_t group, double *out)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (!out || group < 0 || group >= (int)ctx->groups.size()) return fail(ctx, BEC_ERR_INVALID_ARG, "bad axial args");
    bec_status st = check_ready(ctx);
    if (st) return st;
    if ((st = observe_now(ctx))) return st;
    return group_axial_host(ctx, group, out);
}

bec_status bec_render_projections(bec_ctx *ctx, int32_t group, float *xy_a, float *xy_b, float *zy_a, float *zy_b,
                                  float *levels_xy, float *levels_zy)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (group < 0 || group >= (int)ctx->groups.size() || !xy_a || !xy_b || !zy_a || !zy_b)
        return fail(ctx, BEC_ERR_INVALID_ARG, "bad render arguments");
    if (ctx->path != BEC_PATH_FP32_BATCHED) return fail(ctx, BEC_ERR_UNIMPLEMENTED, "rendering needs the batched path");
    bec_status st = check_ready(ctx);
    if (st) return st;
    GroupRec &gr = ctx->groups[group];
    ClassRec &c = ctx->classes[gr.cls];
    cudaStream_t s = ctx->stream;
    if ((st = batched_resolve(ctx, false))) return st;
    const int nxy = c.geom.nx * c.geom.ny, nyz = c.geom.ny * c.geom.nz;
    float *lev = nullptr;
    float4 *rgba = nullptr;
    CKC(cudaMalloc(&lev, sizeof(float) * 2 * (nxy + nyz)));
    if (cudaMalloc(&rgba, sizeof(float4) * 2 * (nxy + nyz)) != cudaSuccess) {
        cudaFree(lev);
        return fail(ctx, BEC_ERR_OUT_OF_MEMORY, "render buffers");
    }
    struct G { float *l; float4 *r; cudaStream_t s; ~G() { cudaStreamSynchronize(s); cudaFree(l); cudaFree(r); } } guard{lev, rgba, s};
    float *lxa = lev, *lxb = lev + nxy, *lza = lev + 2 * nxy, *lzb = lza + nyz;
    CKC(cudaMemsetAsync(lev, 0, sizeof(float) * 2 * (nxy + nyz), s));
    ClassGeom one = c.geom;
    one.n_traj = 1;
    float2 *tx, *ty;
    if ((st = get_tw32(ctx, one.nx, &tx)) || (st = get_tw32(ctx, one.ny, &ty))) return st;
    const float sub = (float)(gr.d.V / (2.0 * gr.d.dV));
    for (int t = 0; t < gr.p.ne; ++t) {
        CKC(cudaMemcpyAsync(ctx->scratch4, c.state + (size_t)(gr.local_first + t) * c.geom.cells,
                            sizeof(float4) * c.geom.cells, cudaMemcpyDeviceToDevice, s));
        fp32_unprep(ctx->scratch4, one, tx, ty, s);
        render_project(ctx->scratch4, one, 1.0f / (float)nxy, sub, lxa, lxb, lza, lzb, s);
    }
    const double scale = 3.0 * gr.d.N * gr.p.ne / ((double)gr.d.cells * gr.d.dV);    // wigner.cu:418
    render_colour(lxa, 2 * nxy, (float)(scale * c.geom.nz), rgba, s);
    render_colour(lza, 2 * nyz, (float)(scale * c.geom.nx), rgba + 2 * nxy, s);
    CKL();
    CKC(cudaMemcpyAsync(xy_a, rgba, sizeof(float4) * nxy, cudaMemcpyDeviceToHost, s));
    CKC(cudaMemcpyAsync(xy_b, rgba + nxy, sizeof(float4) * nxy, cudaMemcpyDeviceToHost, s));
    CKC(cudaMemcpyAsync(zy_a, rgba + 2 * nxy, sizeof(float4) * nyz, cudaMemcpyDeviceToHost, s));
    CKC(cudaMemcpyAsync(zy_b, rgba + 2 * nxy + nyz, sizeof(float4) * nyz, cudaMemcpyDeviceToHost, s));
    if (levels_xy) CKC(cudaMemcpyAsync(levels_xy, lxa, sizeof(float) * 2 * nxy, cudaMemcpyDeviceToHost, s));
    if (levels_zy) CKC(cudaMemcpyAsync(levels_zy, lza, sizeof(float) * 2 * nyz, cudaMemcpyDeviceToHost, s));
    CKC(cudaStreamSynchronize(s));
    return BEC_OK;
}

bec_status bec_run(bec_ctx *ctx, const bec_schedule *sch, bec_moments *samples, double *axial)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (!sch || !samples || sch->n_steps < 0 || sch->sample_every < 0 || (sch->axial && !axial))
        return fail(ctx, BEC_ERR_INVALID_ARG, "bad schedule");
    bec_status st = check_ready(ctx);
    if (st) return st;
    const int n = sch->n_steps;
    const int every = sch->sample_every > 0 ? sch->sample_every : (n > 0 ? n : 1);
    const int n_samples = n / every;
    const size_t ng = ctx->groups.size();
    size_t axial_stride = 0;
    for (auto &g : ctx->groups) axial_stride += (size_t)4 * g.d.nvz;
    double2 pi_m[4];
    rotation(M_PI, 0.0, pi_m);
    if ((st = ensure_plan(ctx))) return st;
    const long long l0 = g_launches;
    CKC(cudaEventRecord(ctx->ev0, ctx->stream));
    int sample = 0;
    auto take_sample = [&]() -> bec_status {
        bec_status st2 = fetch_group_moments(ctx, samples + (size_t)sample * ng);
        if (st2) return st2;
        if (sch->axial) {
            double *dst = axial + (size_t)sample * axial_stride;
            for (size_t g = 0; g < ng; ++g) {
                if ((st2 = group_axial_host(ctx, (int)g, dst))) return st2;
                dst += 4 * ctx->groups[g].d.nvz;
            }
        }
        ++sample;
        return BEC_OK;
    };
    if (ctx->path == BEC_PATH_FP64_PLAIN) {
        for (int i = 1; i <= n; ++i) {
            if ((st = do_evolve(ctx, 1))) return st;
            if (i % every == 0 && sample < n_samples) {
                if ((st = plain_observe(ctx))) return st;
                if ((st = take_sample())) return st;
            }
            if (i == sch->pi_pulse_step && (st = apply_pulse(ctx, pi_m))) return st;
        }
    } else {
        bool obs_due = false;
        // before step j: a sample of the boundary after step j-1, or the pi pulse scheduled there
        auto event_before = [&](int j) {
            return ((j - 1) > 0 && (j - 1) % every == 0 && sample < n_samples) || j - 1 == sch->pi_pulse_step;
        };
        // a moments-only sample between steady steps sums the stored state and leaves the step running;
        // otherwise a pass that ends the step observes the boundary (axial profiles need x-space along z)
        auto sample_boundary = [&]() -> bec_status {
            bec_status st2;
            if (!sch->axial && ctx->pending && !ctx->has_pulse) {
                if ((st2 = batched_moments_stored(ctx))) return st2;
            } else {
                if ((st2 = batched_resolve(ctx, true))) return st2;
                if ((st2 = batched_reduce_obs(ctx))) return st2;
            }
            return take_sample();
        };
        int i = 1;
        while (i <= n) {
            if (obs_due) {
                if ((st = sample_boundary())) return st;
                obs_due = false;
            }
            // a pi pulse scheduled after step i-1 rides on this step's pencil pass (after any sample)
            if (i - 1 == sch->pi_pulse_step && (st = apply_pulse(ctx, pi_m))) return st;
            int len = 1;
            if (ctx->pending && !ctx->has_pulse) {
                // steady steps up to the next sample or pulse: captured graph replays
                while (i + len <= n && !event_before(i + len)) ++len;
                if ((st = run_steady(ctx, len))) return st;
            } else {
                if ((st = batched_step(ctx, ctx->pending ? 0.5f : 0.0f, true))) return st;
                ctx->pending = true;
                ctx->step++;
                ctx->evo_steps++;
            }
            i += len;
            if ((i - 1) % every == 0 && sample < n_samples) obs_due = true;
        }
        if (obs_due && (st = sample_boundary())) return st;
        if (n == sch->pi_pulse_step && (st = apply_pulse(ctx, pi_m))) return st;
    }
    CKC(cudaEventRecord(ctx->ev1, ctx->stream));
    CKC(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->last_ms = ms;
    ctx->last_launches = g_launches - l0;
    return check_step_error(ctx);
}

bec_status bec_observables(const bec_ctx *ctx, int32_t group, const bec_moments *m, bec_obs *out)
{
    if (!ctx || !m || !out || group < 0 || group >= (int)ctx->groups.size()) return BEC_ERR_INVALID_ARG;
    const GroupRec &gr = ctx->groups[group];
    const double ne = gr.p.ne;
    // Wigner term: density subtracts V/(2 dV) per cell (wigner_kernel.cu:283-286), i.e. V/2 per cell after * dV
    const double sub = ne * gr.d.cells * gr.d.V / 2.0;
    const double N1 = m->na - sub, N2 = m->nb - sub;
    out->t = m->t;
    out->N1 = N1 / ne;
    out->N2 = N2 / ne;
    out->Ntotal = (N1 + N2) / ne;
    const double S = std::hypot(m->s_re, m->s_im);
    out->visibility = 2.0 * S / (N1 + N2);
    out->phase = std::atan2(m->s_im, m->s_re);
    double mx = 0.0;
    for (double alpha = 0; alpha < 2 * M_PI; alpha += 0.5) {      // wigner.cu:270
        const double im = std::sin(alpha) * m->s_re + std::cos(alpha) * m->s_im;   // Im(e^{i alpha} S)
        const double n1 = std::fabs((m->na + m->nb) / 2.0 + im - sub);
        const double n2 = std::fabs((m->na + m->nb) / 2.0 - im - sub);
        const double r = (n1 - n2) / (n1 + n2);
        if (std::fabs(r) > mx) mx = std::fabs(r);
    }
    out->visibility_scan = mx;
    return BEC_OK;
}

bec_status bec_phase_scan(const bec_ctx *ctx, int32_t group, const bec_moments *m, int32_t n_alpha,
                          const double *alpha, double *out)
{
    if (!ctx || !m || n_alpha < 0 || (n_alpha > 0 && (!alpha || !out)) || group < 0 ||
        group >= (int)ctx->groups.size())
        return BEC_ERR_INVALID_ARG;
    const GroupRec &gr = ctx->groups[group];
    const double ne = gr.p.ne;
    const double sub = ne * gr.d.cells * gr.d.V / 2.0;
    for (int j = 0; j < n_alpha; ++j) {
        const double im = std::sin(alpha[j]) * m->s_re + std::cos(alpha[j]) * m->s_im;
        out[2 * j] = ((m->na + m->nb) / 2.0 + im - sub) / ne;
        out[2 * j + 1] = ((m->na + m->nb) / 2.0 - im - sub) / ne;
    }
    return BEC_OK;
}

// ------------------------------------------------------------------------ state I/O
bec_status bec_get_state(bec_ctx *ctx, int32_t group, int32_t traj, double *ab)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (!ab || group < 0 || group >= (int)ctx->groups.size()) return fail(ctx, BEC_ERR_INVALID_ARG, "bad args");
    GroupRec &gr = ctx->groups[group];
    if (traj < 0 || traj >= gr.p.ne) return fail(ctx, BEC_ERR_INVALID_ARG, "bad trajectory");
    if (!gr.initialised) return fail(ctx, BEC_ERR_STATE, "group not initialised");
    const int cells = gr.d.cells;
    cudaStream_t s = ctx->stream;
    bec_status st;
    if (ctx->path == BEC_PATH_FP64_PLAIN) {
        CKC(cudaMemcpyAsync(ctx->scratch_a, gr.a + (size_t)traj * cells, sizeof(double2) * cells,
                            cudaMemcpyDeviceToDevice, s));
        CKC(cudaMemcpyAsync(ctx->scratch_b, gr.b + (size_t)traj * cells, sizeof(double2) * cells,
                            cudaMemcpyDeviceToDevice, s));
        if ((st = plain_fft(ctx, ctx->scratch_a, gr.gd, 0))) return st;
        if ((st = plain_fft(ctx, ctx->scratch_b, gr.gd, 0))) return st;
        CKC(cudaMemcpyAsync(ab, ctx->scratch_a, sizeof(double2) * cells, cudaMemcpyDeviceToHost, s));
        CKC(cudaMemcpyAsync(ab + 2 * (size_t)cells, ctx->scratch_b, sizeof(double2) * cells, cudaMemcpyDeviceToHost, s));
        CKC(cudaStreamSynchronize(s));
        return BEC_OK;
    }
    if ((st = batched_resolve(ctx, false))) return st;
    ClassRec &c = ctx->classes[gr.cls];
    CKC(cudaMemcpyAsync(ctx->scratch4, c.state + (size_t)(gr.local_first + traj) * cells, sizeof(float4) * cells,
                        cudaMemcpyDeviceToDevice, s));
    ClassGeom one = c.geom;
    one.n_traj = 1;
    float2 *tx, *ty;
    if ((st = get_tw32(ctx, one.nx, &tx)) || (st = get_tw32(ctx, one.ny, &ty))) return st;
    fp32_unprep(ctx->scratch4, one, tx, ty, s);
    // the stored representation carries the unnormalised x-y inverse transform
    std::vector<float4> h(cells);
    CKC(cudaMemcpyAsync(h.data(), ctx->scratch4, sizeof(float4) * cells, cudaMemcpyDeviceToHost, s));
    CKC(cudaStreamSynchronize(s));
    const double inv = 1.0 / ((double)one.nx * one.ny);
    for (int i = 0; i < cells; ++i) {
        ab[2 * i] = h[i].x * inv; ab[2 * i + 1] = h[i].y * inv;
        ab[2 * ((size_t)cells + i)] = h[i].z * inv; ab[2 * ((size_t)cells + i) + 1] = h[i].w * inv;
    }
    return BEC_OK;
}

bec_status bec_set_state(bec_ctx *ctx, int32_t group, int32_t traj, const double *ab)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (!ab || group < 0 || group >= (int)ctx->groups.size()) return fail(ctx, BEC_ERR_INVALID_ARG, "bad args");
    GroupRec &gr = ctx->groups[group];
    if (traj < 0 || traj >= gr.p.ne) return fail(ctx, BEC_ERR_INVALID_ARG, "bad trajectory");
    const int cells = gr.d.cells;
    cudaStream_t s = ctx->stream;
    bec_status st;
    if (ctx->path == BEC_PATH_FP64_PLAIN) {
        double2 *a = gr.a + (size_t)traj * cells, *b = gr.b + (size_t)traj * cells;
        CKC(cudaMemcpyAsync(a, ab, sizeof(double2) * cells, cudaMemcpyHostToDevice, s));
        CKC(cudaMemcpyAsync(b, ab + 2 * (size_t)cells, sizeof(double2) * cells, cudaMemcpyHostToDevice, s));
        if ((st = plain_fft(ctx, a, gr.gd, 1))) return st;
        if ((st = plain_fft(ctx, b, gr.gd, 1))) return st;
        plain_scale(a, cells, 1.0 / cells, s);
        plain_scale(b, cells, 1.0 / cells, s);
        CKC(cudaStreamSynchronize(s));
        CKL();
        gr.initialised = true;
        return BEC_OK;
    }
    if ((st = batched_resolve(ctx, false))) return st;
    std::vector<float4> h(cells);
    for (int i = 0; i < cells; ++i)
        h[i] = make_float4((float)ab[2 * i], (float)ab[2 * i + 1], (float)ab[2 * ((size_t)cells + i)],
                           (float)ab[2 * ((size_t)cells + i) + 1]);
    ClassRec &c = ctx->classes[gr.cls];
    float4 *dst = c.state + (size_t)(gr.local_first + traj) * cells;
    CKC(cudaMemcpyAsync(dst, h.data(), sizeof(float4) * cells, cudaMemcpyHostToDevice, s));
    ClassGeom one = c.geom;
    one.n_traj = 1;
    float2 *tx, *ty;
    if ((st = get_tw32(ctx, one.nx, &tx)) || (st = get_tw32(ctx, one.ny, &ty))) return st;
    fp32_prep(dst, one, tx, ty, s);
    CKC(cudaStreamSynchronize(s));
    CKL();
    gr.initialised = true;
    return BEC_OK;
}

bec_status bec_profile_steps(bec_ctx *ctx, int32_t n_steps, int32_t max_classes, int32_t *dims, int64_t *traj,
                             double *ms, int32_t *n_classes)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (n_steps < 1 || max_classes < 0 || !n_classes || (max_classes > 0 && (!dims || !traj || !ms)))
        return fail(ctx, BEC_ERR_INVALID_ARG, "bad profile arguments");
    bec_status st = check_ready(ctx);
    if (st) return st;
    cudaStream_t s = ctx->stream;
    const bool plain = ctx->path == BEC_PATH_FP64_PLAIN;
    const int nc = plain ? (int)ctx->groups.size() : (int)ctx->classes.size();
    std::vector<cudaEvent_t> ev;
    struct Destroy { std::vector<cudaEvent_t> &v; ~Destroy() { for (cudaEvent_t e : v) cudaEventDestroy(e); } } destroy{ev};
    auto new_event = [&]() { cudaEvent_t e; cudaEventCreate(&e); ev.push_back(e); return e; };
    // [step][class][pass] -> (start, stop)
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> marks((size_t)n_steps * nc * 2, {nullptr, nullptr});
    for (int i = 0; i < n_steps; ++i) {
        if (plain) {
            for (int g = 0; g < nc; ++g) {
                GroupRec &gr = ctx->groups[g];
                auto &mk = marks[((size_t)i * nc + g) * 2];
                mk.first = new_event();
                mk.second = new_event();
                CKC(cudaEventRecord(mk.first, s));
                for (int t = 0; t < gr.p.ne; ++t)
                    if ((st = plain_step(ctx, gr, t))) return st;
                CKC(cudaEventRecord(mk.second, s));
            }
        } else {
            std::vector<std::pair<cudaEvent_t, cudaEvent_t>> zev(nc), pev(nc);
            for (int c = 0; c < nc; ++c) {
                zev[c] = {new_event(), new_event()};
                pev[c] = {new_event(), new_event()};
                marks[((size_t)i * nc + c) * 2] = zev[c];
                marks[((size_t)i * nc + c) * 2 + 1] = pev[c];
            }
            if ((st = batched_zpass_all(ctx, ctx->pending ? 0.5f : 0.0f, 0.5f, false, nullptr, false, zev.data())))
                return st;
            ctx->pending = true;
            if ((st = batched_ppass_all(ctx, pev.data()))) return st;
        }
        CKL();
        ctx->step++;
        ctx->evo_steps++;
    }
    CKC(cudaStreamSynchronize(s));
    const int nw = std::min(nc, (int)max_classes);
    for (int c = 0; c < nw; ++c) {
        double sum[2] = {0.0, 0.0};
        for (int i = 0; i < n_steps; ++i)
            for (int k = 0; k < 2; ++k) {
                auto &mk = marks[((size_t)i * nc + c) * 2 + k];
                if (!mk.first) continue;
                float t = 0.f;
                cudaEventElapsedTime(&t, mk.first, mk.second);
                sum[k] += t;
            }
        if (plain) {
            const GroupRec &gr = ctx->groups[c];
            dims[3 * c] = gr.d.nvx; dims[3 * c + 1] = gr.d.nvy; dims[3 * c + 2] = gr.d.nvz;
            traj[c] = gr.p.ne;
            ms[2 * c] = sum[0] / n_steps / gr.p.ne;
            ms[2 * c + 1] = 0.0;
        } else {
            const ClassRec &cr = ctx->classes[c];
            dims[3 * c] = cr.geom.nx; dims[3 * c + 1] = cr.geom.ny; dims[3 * c + 2] = cr.geom.nz;
            traj[c] = cr.geom.n_traj;
            ms[2 * c] = sum[0] / n_steps;
            ms[2 * c + 1] = sum[1] / n_steps;
        }
    }
    *n_classes = nc;
    return BEC_OK;
}

int64_t bec_step_index(const bec_ctx *ctx) { return ctx ? ctx->step : -1; }
int64_t bec_evolution_steps(const bec_ctx *ctx) { return ctx ? ctx->evo_steps : -1; }

bec_status bec_profile_fused_step(bec_ctx *ctx, int32_t n_steps, double *ms_per_step, int64_t *cells)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (n_steps < 1 || !ms_per_step || !cells) return fail(ctx, BEC_ERR_INVALID_ARG, "bad arguments");
    if (ctx->path != BEC_PATH_FP32_BATCHED) return fail(ctx, BEC_ERR_STATE, "batched path only");
    bec_status st = check_ready(ctx);
    if (st) return st;
    if ((st = ensure_plan(ctx))) return st;
    if (!ctx->plan.ready) return fail(ctx, BEC_ERR_STATE, "no fused step plan (no register-path grid class)");
    if (!ctx->pending || ctx->has_pulse) {
        if ((st = batched_step(ctx, ctx->pending ? 0.5f : 0.0f, true))) return st;
        ctx->pending = true;
        ctx->step++;
        ctx->evo_steps++;
    }
    double tot = 0.0;
    long long l0 = g_launches;
    for (int i = 0; i < n_steps; ++i) {
        fp32_put_step(ctx->d_step, (uint32_t)ctx->step, ctx->stream);
        if ((st = batched_zpass_all(ctx, 0.5f, 0.5f, false, nullptr, false, nullptr, true))) return st;
        if ((st = batched_ppass_all(ctx, nullptr, false, true))) return st;
        CKC(cudaEventRecord(ctx->ev0, ctx->stream));
        step_launch(ctx->plan, ctx->d_gparams, ctx->d_step, 1.0f, nullptr, ctx->stream);
        CKC(cudaEventRecord(ctx->ev1, ctx->stream));
        CKC(cudaEventSynchronize(ctx->ev1));
        CKL();
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        tot += ms;
        ctx->step++;
        ctx->evo_steps++;
    }
    ctx->last_launches = g_launches - l0;
    long long n = 0;
    for (size_t ci = 0; ci < ctx->classes.size(); ++ci)
        if (ctx->fused[ci]) n += (long long)ctx->classes[ci].geom.n_traj * ctx->classes[ci].geom.cells;
    *ms_per_step = tot / n_steps;
    *cells = n;
    return check_step_error(ctx);
}

bec_status bec_step_plan(bec_ctx *ctx, char *out, int32_t len)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (!out || len < 1) return fail(ctx, BEC_ERR_INVALID_ARG, "null output");
    const std::string d = ctx->path != BEC_PATH_FP32_BATCHED ? std::string("{\"plan\": \"plain path\"}")
                          : ctx->plan_mode == -2 ? std::string("{\"plan\": \"not chosen (no step taken)\"}")
                                                 : ctx->plan_desc;
    if ((int32_t)d.size() >= len) return fail(ctx, BEC_ERR_INVALID_ARG, "output buffer too small");
    std::memcpy(out, d.c_str(), d.size() + 1);
    return BEC_OK;
}

int32_t bec_step_graphs(const bec_ctx *ctx)
{
    if (!ctx || !ctx->use_graphs || ctx->graphs_failed) return 0;
    return (ctx->step_graph[0] ? 1 : 0) + (ctx->step_graph[1] ? 1 : 0);
}
double bec_last_device_ms(const bec_ctx *ctx) { return ctx ? ctx->last_ms : 0.0; }
int64_t bec_last_launch_count(const bec_ctx *ctx) { return ctx ? ctx->last_launches : 0; }

// ---------------------------------------------------------------- checkpoint / resume
namespace {
constexpr uint64_t kCkptMagic = 0x3154504b43454221ull;   // "!BECKPT1" little-endian
constexpr int32_t kCkptVersion = 1;

struct CkptHeader {
    uint64_t magic;
    int32_t version, path, n_groups, pending;
    int64_t n_traj, step, evo_steps, payload;
    int32_t has_pulse, pad;
    double pulse[8];             // pending pulse matrix, row-major (re, im)
};

struct CkptGroup {
    int32_t nvx, nvy, nvz, ne;
    uint64_t seed;
};

size_t ckpt_payload(const bec_ctx *ctx)
{
    size_t n = 0;
    if (ctx->path == BEC_PATH_FP64_PLAIN)
        for (auto &gr : ctx->groups) n += 2 * sizeof(double2) * (size_t)gr.p.ne * gr.d.cells;
    else
        for (auto &c : ctx->classes) n += sizeof(float4) * (size_t)c.geom.n_traj * c.geom.cells;
    return n;
}

size_t ckpt_bytes(const bec_ctx *ctx)
{
    return sizeof(CkptHeader) + sizeof(CkptGroup) * ctx->groups.size() + ckpt_payload(ctx);
}
} // namespace

int64_t bec_checkpoint_bytes(const bec_ctx *ctx) { return ctx ? (int64_t)ckpt_bytes(ctx) : 0; }

bec_status bec_checkpoint_save(bec_ctx *ctx, void *buf, int64_t bytes)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (!buf || bytes < (int64_t)ckpt_bytes(ctx)) return fail(ctx, BEC_ERR_INVALID_ARG, "checkpoint buffer too small");
    bec_status st = check_ready(ctx);
    if (st) return st;
    char *p = static_cast<char *>(buf);
    CkptHeader h{};
    h.magic = kCkptMagic;
    h.version = kCkptVersion;
    h.path = ctx->path;
    h.n_groups = (int32_t)ctx->groups.size();
    h.pending = ctx->pending ? 1 : 0;
    h.n_traj = ctx->n_traj;
    h.step = ctx->step;
    h.evo_steps = ctx->evo_steps;
    h.payload = (int64_t)ckpt_payload(ctx);
    h.has_pulse = ctx->has_pulse ? 1 : 0;
    for (int i = 0; i < 4; ++i) { h.pulse[2 * i] = ctx->pulse[i].x; h.pulse[2 * i + 1] = ctx->pulse[i].y; }
    std::memcpy(p, &h, sizeof h);
    p += sizeof h;
    for (auto &gr : ctx->groups) {
        CkptGroup g{gr.d.nvx, gr.d.nvy, gr.d.nvz, gr.p.ne, gr.p.seed};
        std::memcpy(p, &g, sizeof g);
        p += sizeof g;
    }
    // the stored device representation, bit for bit (the batched path's pending half kick and pulse stay
    // pending, so a resumed run merges them into its next pencil pass exactly as this one would)
    if (ctx->path == BEC_PATH_FP64_PLAIN) {
        for (auto &gr : ctx->groups) {
            const size_t n = sizeof(double2) * (size_t)gr.p.ne * gr.d.cells;
            CKC(cudaMemcpyAsync(p, gr.a, n, cudaMemcpyDeviceToHost, ctx->stream));
            CKC(cudaMemcpyAsync(p + n, gr.b, n, cudaMemcpyDeviceToHost, ctx->stream));
            p += 2 * n;
        }
    } else {
        for (auto &c : ctx->classes) {
            const size_t n = sizeof(float4) * (size_t)c.geom.n_traj * c.geom.cells;
            if (n) CKC(cudaMemcpyAsync(p, c.state, n, cudaMemcpyDeviceToHost, ctx->stream));
            p += n;
        }
    }
    CKC(cudaStreamSynchronize(ctx->stream));
    return BEC_OK;
}

bec_status bec_checkpoint_load(bec_ctx *ctx, const void *buf, int64_t bytes)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (!buf || bytes < (int64_t)sizeof(CkptHeader)) return fail(ctx, BEC_ERR_INVALID_ARG, "checkpoint too short");
    const char *p = static_cast<const char *>(buf);
    CkptHeader h;
    std::memcpy(&h, p, sizeof h);
    p += sizeof h;
    if (h.magic != kCkptMagic || h.version != kCkptVersion)
        return fail(ctx, BEC_ERR_INVALID_ARG, "not a checkpoint of this library");
    if (h.path != ctx->path || h.n_groups != (int32_t)ctx->groups.size() || h.n_traj != ctx->n_traj ||
        h.payload != (int64_t)ckpt_payload(ctx) || bytes < (int64_t)ckpt_bytes(ctx) || h.step < 0 || h.evo_steps < 0)
        return fail(ctx, BEC_ERR_INVALID_ARG, "checkpoint of a different context layout");
    for (auto &gr : ctx->groups) {
        CkptGroup g;
        std::memcpy(&g, p, sizeof g);
        p += sizeof g;
        if (g.nvx != gr.d.nvx || g.nvy != gr.d.nvy || g.nvz != gr.d.nvz || g.ne != gr.p.ne || g.seed != gr.p.seed)
            return fail(ctx, BEC_ERR_INVALID_ARG, "checkpoint group differs in grid, trajectories or seed");
    }
    if (ctx->path == BEC_PATH_FP64_PLAIN) {
        for (auto &gr : ctx->groups) {
            const size_t n = sizeof(double2) * (size_t)gr.p.ne * gr.d.cells;
            CKC(cudaMemcpyAsync(gr.a, p, n, cudaMemcpyHostToDevice, ctx->stream));
            CKC(cudaMemcpyAsync(gr.b, p + n, n, cudaMemcpyHostToDevice, ctx->stream));
            p += 2 * n;
        }
    } else {
        for (auto &c : ctx->classes) {
            const size_t n = sizeof(float4) * (size_t)c.geom.n_traj * c.geom.cells;
            if (n) CKC(cudaMemcpyAsync(c.state, p, n, cudaMemcpyHostToDevice, ctx->stream));
            p += n;
        }
    }
    CKC(cudaStreamSynchronize(ctx->stream));
    ctx->step = h.step;
    ctx->evo_steps = h.evo_steps;
    ctx->pending = h.pending != 0;
    ctx->has_pulse = h.has_pulse != 0;
    for (int i = 0; i < 4; ++i) ctx->pulse[i] = make_double2(h.pulse[2 * i], h.pulse[2 * i + 1]);
    for (auto &gr : ctx->groups) gr.initialised = true;
    return BEC_OK;
}

bec_status bec_set_step_index(bec_ctx *ctx, int64_t step, int64_t evo_steps)
{
    if (!ctx) return BEC_ERR_INVALID_ARG;
    if (step < 0 || evo_steps < 0 || step > 0xFFFFFFFFll)
        return fail(ctx, BEC_ERR_INVALID_ARG, "step index out of range");
    ctx->step = step;
    ctx->evo_steps = evo_steps;
    return BEC_OK;
}

} // extern "C"
