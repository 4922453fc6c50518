// mom6b_api.cu -- the model object and the high-level C ABI (include/mom6b.h).
//
// A model keeps the whole state of rk2_serial_driver resident in HBM and
// advances it with the fused kernels of this directory.  One split RK2
// iteration (rk2_serial_driver.F90:218-399) is enqueued as
//
//   predictor   k_tendency(u, v, h0 -> up, vp)        transports+hor_visc+CorAdCalc+update
//               k_vertvisc(up, vp; h0)                 vert_visc_coef + vert_visc_apply
//               k_ppm_edges + k_cont_faces(up, h0 -> hB)  continuity_PPM
//   corrector   k_tendency(up, vp, hB -> u, v)
//               k_vertvisc(u, v; hB)
//               k_ppm_edges + k_cont_faces(u, hB -> hA)
//   barotropic  k_btstep(eta, ubt, vbt -> ubt_av, vbt_av, eta_av)
//               k_btstep(eta_av, ubt_av, vbt_av -> ubt_av, vbt_av, eta)
//
// The reset h <- h0 at the top of the reference iteration is realised by
// reading h0 directly in the predictor; the thickness ping-pongs between hB
// (after the predictor, the reference's htmp) and hA (the state h), whose
// halo ring is h0 unless the halo fill is enabled.  The barotropic chain
// reads nothing the 3-D chain writes (in rk2_serial_driver.F90:218-399 btstep
// only sees eta/ubt/vbt), so it can run on a second stream joined by events.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mom6b.h"
#include "diag.h"
#include "host_init.h"
#include "hor_visc.h"
#include "kernels.h"
#include "mlp.h"


using namespace mom6b;

static thread_local std::string g_last_error;

static int fail(int code, const std::string& msg)
{
    g_last_error = msg;
    return code;
}

int mom6b_internal_fail(int code, const std::string& msg) { return fail(code, msg); }

#define CK(call)                                                                     \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess)                                                       \
            return fail(MOM6B_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct TimedLaunch {
    std::string name;
    cudaEvent_t a, b;
};

struct mom6b_model {
    mom6b_config cfg;
    std::unique_ptr<HostGrid> grid;
    Dims D;
    Metrics M;
    UniMetrics U{};
    std::vector<void*> allocs;
    // state
    double *u, *v, *hA, *hB, *h0, *up, *vp, *uh, *hW, *hE, *uhbt0, *uh_ovl;
    double *eta, *ubt, *vbt, *ubt_av, *vbt_av, *eta_av;
    double *h_u, *FA_u_W0, *FA_u_WW, *FA_u_E0, *FA_u_EE, *uBT_WW, *uBT_EE, *du_cor;
    double *taux_bot, *tauy_bot;
    double *taux, *tauy, *Ray_u, *Ray_v;
    unsigned char *ray_layer_u, *ray_layer_v;
    BTWork bt;
    cudaStream_t s3d = nullptr, s2d = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int64_t launches = 0;
    int64_t launches_per_step = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    bool overlap_bt = false;
    // set by mom6b_step_host_io for one eager step: the barotropic chain on
    // s2d, which the caller has already forked from s3d
    bool split_bt = false;
    bool timing = false;
    int stall_test = 0;   // BTParams::stall_test of the step's barotropic loops
    std::vector<TimedLaunch> pending;
    std::map<std::string, std::pair<double, int64_t>> timed;  // ms total, launches
    // learned barotropic surrogate (k_mlp.cu): the network, whether it
    // replaces btstep, the shadow check (every sur_every steps the plain loop
    // runs from the same state and checks the surrogate's eta) and its record
    std::unique_ptr<Mlp> sur;
    bool sur_on = false, sur_fallen = false;
    int sur_every = 10;
    double sur_thresh = 1.0e-3;
    int64_t sur_steps = 0, sur_checks = 0, sur_fallbacks = 0;
    double sur_last_err = 0.0, sur_max_err = 0.0;
    double sur_loss_first = 0.0, sur_loss_last = 0.0, sur_train_s = 0.0;
    int64_t sur_train_steps = 0;
    double *sh_eta = nullptr, *sh_ubt_av = nullptr, *sh_vbt_av = nullptr, *sh_eta_av = nullptr;
    double* sur_acc = nullptr;
    // barotropic state of the training and evaluation runs
    double *tr_e = nullptr, *tr_u = nullptr, *tr_v = nullptr;
    double *tr_ea = nullptr, *tr_ua = nullptr, *tr_va = nullptr;
    // diagnostics (mom6_diag.F90) and the driver's four fields
    std::unique_ptr<DiagCtrl> diag;
    bool diag_driver = false;
    int id_KE = -1, id_diffu_sum = -1, id_diffv_sum = -1, id_mass = -1;
    double *dg_du = nullptr, *dg_dv = nullptr, *dg_ke = nullptr, *dg_mass = nullptr;
    // Coriolis scheme of the tendency (1 SADOURNY75_ENERGY, 2 ARAKAWA_HSU90, 3 ARAKAWA_LAMB81)
    int cor_scheme = 1;
    // meridional continuity: intermediate thickness, vh, h_v, BT_cont's v fields
    bool merid = false;
    double *hZ = nullptr, *vh = nullptr, *h_v = nullptr, *vh_ovl = nullptr;
    double *FA_v_S0 = nullptr, *FA_v_SS = nullptr, *FA_v_N0 = nullptr, *FA_v_NN = nullptr;
    double *vBT_SS = nullptr, *vBT_NN = nullptr, *dv_cor = nullptr;
    // vertical-viscosity remnant (vert_visc_remnant) written by every
    // vertvisc and read by the continuity that follows it
    bool remnant = false;
    double *visc_rem_u = nullptr, *visc_rem_v = nullptr;
    // hor_visc scheme branches (mom6b_set_hor_visc): the general kernel's
    // parameters and arrays, and the accelerations it hands to the tendency
    bool hvgen = false;
    HorViscGen hvp{};
    double *hv_du = nullptr, *hv_dv = nullptr;
    // the halo exchange of a decomposed run (mom6b_set_exchange)
    mom6b_exchange_fn xfn = nullptr;
    void* xctx = nullptr;
};

static double* dalloc(mom6b_model* m, size_t n, cudaError_t* err)
{
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, n * sizeof(double) + 16);
    if (e != cudaSuccess) { *err = e; return nullptr; }
    cudaMemset(p, 0, n * sizeof(double) + 16);
    m->allocs.push_back(p);
    return (double*)p;
}

static void free_all(mom6b_model* m)
{
    for (void* p : m->allocs) cudaFree(p);
    m->allocs.clear();
    for (auto& t : m->pending) { cudaEventDestroy(t.a); cudaEventDestroy(t.b); }
    m->pending.clear();
    if (m->graph_exec) cudaGraphExecDestroy(m->graph_exec);
    if (m->graph) cudaGraphDestroy(m->graph);
    if (m->ev_fork) cudaEventDestroy(m->ev_fork);
    if (m->ev_join) cudaEventDestroy(m->ev_join);
    if (m->s3d) cudaStreamDestroy(m->s3d);
    if (m->s2d) cudaStreamDestroy(m->s2d);
}

extern "C" const char* mom6b_last_error(void) { return g_last_error.c_str(); }
extern "C" const char* mom6b_version(void) { return "mom6b 0.1 (sm_100a)"; }

extern "C" int mom6b_config_default(mom6b_config* c, int init_mode)
{
    if (!c) return fail(MOM6B_ERR_ARG, "null config");
    std::memset(c, 0, sizeof(*c));
    c->ni = 180; c->nj = 180; c->nk = 75; c->bt_nsteps = 30;
    c->init_mode = init_mode;
    c->dx_km = 10.0; c->lat_deg = 45.0;
    c->Kv = 1.0e-4; c->Kv_ml = 1.0e-2; c->Kv_extra_bbl = 1.0e-2;
    c->Hmix = 50.0; c->Hbbl = 10.0;
    c->precision = MOM6B_FP64;
    c->use_graph = 0;
    if (init_mode == MOM6B_INIT_REF) {
        c->dt = 300.0; c->Kh = 100.0; c->bc_fill = 0;
    } else if (init_mode == MOM6B_INIT_CFG) {
        c->dt = 600.0; c->Kh = 1.0e3; c->bc_fill = 1;
    } else {
        return fail(MOM6B_ERR_ARG, "unknown init mode");
    }
    return MOM6B_OK;
}

template <class T>
static int upload(T* dst, const std::vector<T>& src)
{
    CK(cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    return MOM6B_OK;
}

static int set_ray_flags(mom6b_model* m, const std::vector<double>& Ru,
                         const std::vector<double>& Rv)
{
    const HostGrid& g = *m->grid;
    std::vector<unsigned char> fu(g.nk, 0), fv(g.nk, 0);
    for (int k = 0; k < g.nk; ++k) {
        const double* pu = Ru.data() + (size_t)k * g.plane;
        const double* pv = Rv.data() + (size_t)k * g.plane;
        for (size_t q = 0; q < g.plane; ++q) {
            if (pu[q] != 0.0) fu[k] = 1;
            if (pv[q] != 0.0) fv[k] = 1;
        }
    }
    CK(cudaMemcpy(m->ray_layer_u, fu.data(), g.nk, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(m->ray_layer_v, fv.data(), g.nk, cudaMemcpyHostToDevice));
    return MOM6B_OK;
}

static bool IareaT_uniform(const HostGrid& g)
{
    for (const std::vector<double>* a : {&g.IareaT, &g.IdxCu, &g.IdyCv}) {
        double v0 = (*a)[g.at(1, 1)];
        for (int j = 1; j <= g.n2 - 1; ++j)
            for (int i = 1; i <= g.n1 - 1; ++i)
                if ((*a)[g.at(i, j)] != v0) return false;
    }
    return true;
}

// The uniform-metric kernels apply when every metric the step reads is one
// value over the points the kernels touch ([1, n1-1] x [1, n2-1]) and
// CoriolisBu depends on j only.
static int detect_uniform(mom6b_model* m)
{
    const HostGrid& g = *m->grid;
    UniMetrics& U = m->U;
    U.valid = 0;
    U.valid_bt = 0;
    if (m->cfg.general_metrics) return MOM6B_OK;
    bool ok = true;
    auto uni = [&](const std::vector<double>& a, double* out) {
        double v0 = a[g.at(1, 1)];
        for (int j = 1; j <= g.n2 - 1 && ok; ++j)
            for (int i = 1; i <= g.n1 - 1; ++i)
                if (a[g.at(i, j)] != v0) { ok = false; break; }
        *out = v0;
    };
    uni(g.IareaT, &U.IareaT); uni(g.areaT, &U.areaT); uni(g.dxT, &U.dxT);
    uni(g.IdxT, &U.IdxT); uni(g.dxCu, &U.dxCu); uni(g.dyCu, &U.dyCu);
    uni(g.dy_Cu, &U.dy_Cu); uni(g.IdxCu, &U.IdxCu); uni(g.IdyCu, &U.IdyCu);
    uni(g.dxCv, &U.dxCv); uni(g.dyCv, &U.dyCv); uni(g.IdxCv, &U.IdxCv);
    uni(g.IdyCv, &U.IdyCv); uni(g.IareaBu, &U.IareaBu); uni(g.IareaCu, &U.IareaCu);
    uni(g.IareaCv, &U.IareaCv); uni(g.mask2dT, &U.mask2dT); uni(g.mask2dBu, &U.mask2dBu);
    uni(g.mask2dCu, &U.mask2dCu); uni(g.mask2dCv, &U.mask2dCv); uni(g.Area_q, &U.Area_q);
    uni(g.DX_dyT, &U.DX_dyT); uni(g.DY_dxT, &U.DY_dxT); uni(g.DX_dyBu, &U.DX_dyBu);
    uni(g.DY_dxBu, &U.DY_dxBu); uni(g.dx2h, &U.dx2h); uni(g.dy2h, &U.dy2h);
    uni(g.dx2q, &U.dx2q); uni(g.dy2q, &U.dy2q); uni(g.red_xx, &U.red_xx);
    uni(g.red_xy, &U.red_xy); uni(g.Kh_xx, &U.Kh_xx); uni(g.Kh_xy, &U.Kh_xy);
    std::vector<double> cor(g.n2);
    for (int j = 1; j <= g.n2 && ok; ++j) {
        cor[j - 1] = g.CoriolisBu[g.at(1, j)];
        for (int i = 1; i <= g.n1; ++i)
            if (g.CoriolisBu[g.at(i, j)] != cor[j - 1]) { ok = false; break; }
    }
    // barotropic metrics, checked separately
    bool okb = true;
    auto unib = [&](const std::vector<double>& a, double* out) {
        double v0 = a[g.at(1, 1)];
        for (int j = 1; j <= g.n2 - 1 && okb; ++j)
            for (int i = 1; i <= g.n1 - 1; ++i)
                if (a[g.at(i, j)] != v0) { okb = false; break; }
        *out = v0;
    };
    unib(g.Datu, &U.Datu); unib(g.Datv, &U.Datv); unib(g.gtot_E, &U.gtot_E);
    unib(g.gtot_W, &U.gtot_W); unib(g.gtot_N, &U.gtot_N); unib(g.gtot_S, &U.gtot_S);
    unib(g.bt_rem_u, &U.bt_rem_u); unib(g.bt_rem_v, &U.bt_rem_v);
    std::vector<double> f4u(4 * (size_t)g.n2), f4v(4 * (size_t)g.n2);
    for (int j = 1; j <= g.n2 && okb; ++j)
        for (int c = 0; c < 4 && okb; ++c) {
            f4u[(j - 1) * 4 + c] = g.f_4_u[4 * g.at(1, j) + c];
            f4v[(j - 1) * 4 + c] = g.f_4_v[4 * g.at(1, j) + c];
            for (int i = 1; i <= g.n1; ++i)
                if (g.f_4_u[4 * g.at(i, j) + c] != f4u[(j - 1) * 4 + c] ||
                    g.f_4_v[4 * g.at(i, j) + c] != f4v[(j - 1) * 4 + c]) { okb = false; break; }
        }
    cudaError_t err = cudaSuccess;
    if (ok) {
        double* d = dalloc(m, g.n2, &err);
        if (!d) return fail(MOM6B_ERR_NOMEM, "device allocation failed");
        CK(cudaMemcpy(d, cor.data(), g.n2 * sizeof(double), cudaMemcpyHostToDevice));
        U.cor_row = d;
        U.valid = 1;
        // the fast tendency's products of the uniform metrics
        TendFold& K = U.tf;
        const double mB = U.mask2dBu;
        K.kRv = mB * U.dyCv * U.IareaBu;
        K.kRu = mB * U.dxCu * U.IareaBu;
        K.kQn = 2.0 * U.Area_q / U.areaT;
        K.kQe = 2.0e-20 / U.areaT;
        K.kSv = -0.25 * U.Kh_xy * mB * mB * U.red_xy * U.DY_dxBu * U.IdyCv;
        K.kSu = -0.25 * U.Kh_xy * mB * mB * U.red_xy * U.DX_dyBu * U.IdxCu;
        K.kKu = 0.25 * U.dyCu / U.areaT;
        K.kKv = 0.25 * U.dxCv / U.areaT;
        K.kXu = U.Kh_xx * U.red_xx * U.DY_dxT * U.IdyCu;
        K.kXv = U.Kh_xx * U.red_xx * U.DX_dyT * U.IdxCv;
        K.kTu = 0.5 * U.dyCu;
        K.kTv = 0.5 * U.dxCv;
        K.kCu = 0.25 * U.IdxCu;
        K.kCv = 0.25 * U.IdyCv;
        K.kHm = 0.5 * U.mask2dT;
        K.kDq = U.IdxCu * U.dx2q * U.IareaCu;
        K.kDh = U.IdyCu * U.dy2h * U.IareaCu;
        K.kEq = U.IdyCv * U.dy2q * U.IareaCv;
        K.kEh = U.IdxCv * U.dx2h * U.IareaCv;
    }
    if (okb && IareaT_uniform(g)) {
        double* du = dalloc(m, 4 * (size_t)g.n2, &err);
        double* dv = dalloc(m, 4 * (size_t)g.n2, &err);
        if (!du || !dv) return fail(MOM6B_ERR_NOMEM, "device allocation failed");
        CK(cudaMemcpy(du, f4u.data(), f4u.size() * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dv, f4v.data(), f4v.size() * sizeof(double), cudaMemcpyHostToDevice));
        U.f4u_row = du;
        U.f4v_row = dv;
        U.IareaT = g.IareaT[g.at(1, 1)];
        U.IdxCu = g.IdxCu[g.at(1, 1)];
        U.IdyCv = g.IdyCv[g.at(1, 1)];
        U.valid_bt = 1;
    }
    return MOM6B_OK;
}

extern "C" int mom6b_create(const mom6b_config* cfg, mom6b_model** out)
{
    if (!cfg || !out) return fail(MOM6B_ERR_ARG, "null argument");
    *out = nullptr;
    if (cfg->ni < 8 || cfg->nj < 8 || cfg->nk < 2 || cfg->bt_nsteps < 1)
        return fail(MOM6B_ERR_ARG, "sizes must satisfy ni, nj >= 8, nk >= 2, bt_nsteps >= 1");
    if (cfg->nk > 1024) return fail(MOM6B_ERR_ARG, "nk > 1024 not supported");
    if ((long long)(cfg->ni + 2) * (cfg->nj + 2) > (1LL << 30))
        return fail(MOM6B_ERR_ARG, "horizontal grid too large");
    if (cfg->precision != MOM6B_FP64 && cfg->precision != MOM6B_MIXED)
        return fail(MOM6B_ERR_ARG, "unknown precision");
    {
        const int gni = cfg->ni_global > 0 ? cfg->ni_global : cfg->ni;
        const int gnj = cfg->nj_global > 0 ? cfg->nj_global : cfg->nj;
        if (cfg->i_offset < 0 || cfg->j_offset < 0 || cfg->i_offset + (cfg->ni - 4) > gni - 4 ||
            cfg->j_offset + (cfg->nj - 4) > gnj - 4 || (cfg->cuts & ~15))
            return fail(MOM6B_ERR_ARG, "subdomain outside the global domain");
        if (cfg->cuts && (cfg->bc_fill || cfg->precision != MOM6B_FP64))
            return fail(MOM6B_ERR_ARG, "a subdomain with cuts steps in FP64 without halo fill");
    }
    CK(cudaSetDevice(cfg->device));

    auto m = std::make_unique<mom6b_model>();
    m->cfg = *cfg;
    m->grid = std::make_unique<HostGrid>(*cfg);
    HostGrid& g = *m->grid;
    g.build();
    Dims& D = m->D;
    D.n1 = g.n1; D.n2 = g.n2; D.nk = g.nk;
    D.is = g.is; D.ie = g.ie; D.js = g.js; D.je = g.je;
    D.isd = g.isd; D.ied = g.ied; D.jsd = g.jsd; D.jed = g.jed;
    D.plane = (long long)g.plane;
    D.cw = (cfg->cuts & MOM6B_CUT_W) != 0; D.ce = (cfg->cuts & MOM6B_CUT_E) != 0;
    D.cs = (cfg->cuts & MOM6B_CUT_S) != 0; D.cn = (cfg->cuts & MOM6B_CUT_N) != 0;

    const size_t n2 = g.plane, n3 = g.plane * (size_t)g.nk;
    cudaError_t err = cudaSuccess;
    auto A2 = [&]() { return dalloc(m.get(), n2, &err); };
    auto A3 = [&]() { return dalloc(m.get(), n3, &err); };
    // metrics
    struct Up { const double** dst; const std::vector<double>* src; };
    double* dm[64];
    int nm = 0;
    std::vector<Up> ups = {
        {&m->M.IareaT, &g.IareaT}, {&m->M.areaT, &g.areaT}, {&m->M.dxT, &g.dxT},
        {&m->M.IdxT, &g.IdxT}, {&m->M.dxCu, &g.dxCu}, {&m->M.dyCu, &g.dyCu},
        {&m->M.dy_Cu, &g.dy_Cu}, {&m->M.IdxCu, &g.IdxCu}, {&m->M.IdyCu, &g.IdyCu},
        {&m->M.dxCv, &g.dxCv}, {&m->M.dyCv, &g.dyCv}, {&m->M.IdxCv, &g.IdxCv},
        {&m->M.IdyCv, &g.IdyCv}, {&m->M.IareaBu, &g.IareaBu},
        {&m->M.CoriolisBu, &g.CoriolisBu}, {&m->M.IareaCu, &g.IareaCu},
        {&m->M.IareaCv, &g.IareaCv}, {&m->M.mask2dT, &g.mask2dT},
        {&m->M.mask2dBu, &g.mask2dBu}, {&m->M.mask2dCu, &g.mask2dCu},
        {&m->M.mask2dCv, &g.mask2dCv}, {&m->M.Area_q, &g.Area_q},
        {&m->M.DX_dyT, &g.DX_dyT}, {&m->M.DY_dxT, &g.DY_dxT},
        {&m->M.DX_dyBu, &g.DX_dyBu}, {&m->M.DY_dxBu, &g.DY_dxBu},
        {&m->M.dx2h, &g.dx2h}, {&m->M.dy2h, &g.dy2h}, {&m->M.dx2q, &g.dx2q},
        {&m->M.dy2q, &g.dy2q}, {&m->M.red_xx, &g.red_xx}, {&m->M.red_xy, &g.red_xy},
        {&m->M.Kh_xx, &g.Kh_xx}, {&m->M.Kh_xy, &g.Kh_xy}, {&m->M.Datu, &g.Datu},
        {&m->M.Datv, &g.Datv}, {&m->M.gtot_E, &g.gtot_E}, {&m->M.gtot_W, &g.gtot_W},
        {&m->M.gtot_N, &g.gtot_N}, {&m->M.gtot_S, &g.gtot_S},
        {&m->M.bt_rem_u, &g.bt_rem_u}, {&m->M.bt_rem_v, &g.bt_rem_v},
        {&m->M.dyT, &g.dyT}, {&m->M.IdyT, &g.IdyT}};
    for (auto& up : ups) {
        double* p = A2();
        if (!p) return fail(MOM6B_ERR_NOMEM, "device allocation failed");
        *up.dst = p;
        int rc = upload(p, *up.src);
        if (rc) return rc;
        dm[nm++ % 64] = p;
    }
    {
        double* p4u = dalloc(m.get(), 4 * n2, &err);
        double* p4v = dalloc(m.get(), 4 * n2, &err);
        if (!p4u || !p4v) return fail(MOM6B_ERR_NOMEM, "device allocation failed");
        if (int rc = upload(p4u, g.f_4_u)) return rc;
        if (int rc = upload(p4v, g.f_4_v)) return rc;
        m->M.f_4_u = p4u; m->M.f_4_v = p4v;
    }
    m->taux = A2(); m->tauy = A2(); m->Ray_u = A3(); m->Ray_v = A3();
    {
        void* pf = nullptr;
        if (cudaMalloc(&pf, 2 * (size_t)g.nk + 32) != cudaSuccess)
            return fail(MOM6B_ERR_NOMEM, "device allocation failed");
        m->allocs.push_back(pf);
        m->ray_layer_u = (unsigned char*)pf;
        m->ray_layer_v = (unsigned char*)pf + g.nk;
    }
    // state and outputs
    m->u = A3(); m->v = A3(); m->hA = A3(); m->hB = A3(); m->h0 = A3();
    m->up = A3(); m->vp = A3(); m->uh = A3(); m->hW = A3(); m->hE = A3();
    m->h_u = A3();
    m->uh_ovl = dalloc(m.get(), continuity_overlap_doubles(m->D), &err);
    m->uhbt0 = A2();
    m->eta = A2(); m->ubt = A2(); m->vbt = A2(); m->ubt_av = A2(); m->vbt_av = A2();
    m->eta_av = A2();
    m->FA_u_W0 = A2(); m->FA_u_WW = A2(); m->FA_u_E0 = A2(); m->FA_u_EE = A2();
    m->uBT_WW = A2(); m->uBT_EE = A2(); m->du_cor = A2();
    m->taux_bot = A2(); m->tauy_bot = A2();
    BTWork& W = m->bt;
    W.eta = A2(); W.eta_pred = A2(); W.ubt = A2(); W.vbt = A2(); W.ubt_prev = A2();
    W.vbt_prev = A2(); W.uhbt = A2(); W.vhbt = A2(); W.PFu = A2(); W.PFv = A2();
    W.ubt_av = A2(); W.vbt_av = A2();
    {
        void* pb = nullptr;
        const size_t nb = 64 + kBtMaxTiles * sizeof(unsigned int);
        if (cudaMalloc(&pb, nb) != cudaSuccess) return fail(MOM6B_ERR_NOMEM, "device allocation failed");
        cudaMemset(pb, 0, nb);
        m->allocs.push_back(pb);
        W.bar_count = (unsigned int*)pb;
        W.bar_gen = (unsigned int*)pb + 4;
        W.status = (int*)pb + 8;
        W.tile_flag = (unsigned int*)pb + 16;
    }
    if (err != cudaSuccess || !m->u || !W.vbt_av)
        return fail(MOM6B_ERR_NOMEM, std::string("device allocation failed: ") + cudaGetErrorString(err));
    m->M.taux = m->taux; m->M.tauy = m->tauy; m->M.Ray_u = m->Ray_u; m->M.Ray_v = m->Ray_v;
    if (int rc = detect_uniform(m.get())) return rc;
    m->M.ray_layer_u = m->ray_layer_u; m->M.ray_layer_v = m->ray_layer_v;

    // initial state
    {
        std::vector<double> u, v, h0, eta, ubt, vbt, Ru, Rv;
        g.initial_state(u, v, h0, eta, ubt, vbt);
        g.rayleigh(Ru, Rv);
        if (cfg->precision == MOM6B_MIXED) {
            // 3-D state stored as FP32 in the same buffers
            auto upf = [&](double* dst, const std::vector<double>& src) -> int {
                std::vector<float> f(src.begin(), src.end());
                CK(cudaMemcpy(dst, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
                return MOM6B_OK;
            };
            if (int rc = upf(m->u, u)) return rc;
            if (int rc = upf(m->v, v)) return rc;
            if (int rc = upf(m->h0, h0)) return rc;
            if (int rc = upf(m->hA, h0)) return rc;
            if (int rc = upf(m->hB, h0)) return rc;
        } else {
            if (int rc = upload(m->u, u)) return rc;
            if (int rc = upload(m->v, v)) return rc;
            if (int rc = upload(m->h0, h0)) return rc;
            if (int rc = upload(m->hA, h0)) return rc;
            if (int rc = upload(m->hB, h0)) return rc;
        }
        if (int rc = upload(m->eta, eta)) return rc;
        if (int rc = upload(m->ubt, ubt)) return rc;
        if (int rc = upload(m->vbt, vbt)) return rc;
        if (int rc = upload(m->taux, g.taux)) return rc;
        if (int rc = upload(m->tauy, g.tauy)) return rc;
        if (int rc = upload(m->Ray_u, Ru)) return rc;
        if (int rc = upload(m->Ray_v, Rv)) return rc;
        if (int rc = set_ray_flags(m.get(), Ru, Rv)) return rc;
    }
    CK(cudaStreamCreateWithFlags(&m->s3d, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&m->s2d, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&m->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&m->ev_join, cudaEventDisableTiming));
    if (cfg->bc_fill) {
        const Dims& Dd = m->D;
        if (cfg->precision == MOM6B_MIXED) {
            CK(launch_halo_fill_f(Dd, (float*)m->h0, g.nk, 0, m->s3d));
            CK(launch_halo_fill_f(Dd, (float*)m->hA, g.nk, 0, m->s3d));
            CK(launch_halo_fill_f(Dd, (float*)m->hB, g.nk, 0, m->s3d));
            CK(launch_halo_fill_f(Dd, (float*)m->u, g.nk, 1, m->s3d));
            CK(launch_halo_fill_f(Dd, (float*)m->v, g.nk, 2, m->s3d));
        } else {
            CK(launch_halo_fill(Dd, m->h0, g.nk, 0, m->s3d));
            CK(launch_halo_fill(Dd, m->hA, g.nk, 0, m->s3d));
            CK(launch_halo_fill(Dd, m->hB, g.nk, 0, m->s3d));
            CK(launch_halo_fill(Dd, m->u, g.nk, 1, m->s3d));
            CK(launch_halo_fill(Dd, m->v, g.nk, 2, m->s3d));
        }
        CK(launch_halo_fill(Dd, m->eta, 1, 0, m->s3d));
        CK(launch_halo_fill(Dd, m->ubt, 1, 1, m->s3d));
        CK(launch_halo_fill(Dd, m->vbt, 1, 2, m->s3d));
    }
    CK(cudaStreamSynchronize(m->s3d));
    *out = m.release();
    return MOM6B_OK;
}

extern "C" int mom6b_destroy(mom6b_model* m)
{
    if (!m) return MOM6B_OK;
    if (m->s3d) cudaStreamSynchronize(m->s3d);
    if (m->s2d) cudaStreamSynchronize(m->s2d);
    free_all(m);
    delete m;
    return MOM6B_OK;
}

// launch bookkeeping: count every kernel and optionally time it
template <class F>
static cudaError_t timed(mom6b_model* m, cudaStream_t s, const char* name, F&& launch)
{
    TimedLaunch t;
    if (m->timing) {
        t.name = name;
        cudaEventCreate(&t.a);
        cudaEventCreate(&t.b);
        cudaEventRecord(t.a, s);
    }
    cudaError_t e = launch();
    ++m->launches;
    if (m->timing) {
        cudaEventRecord(t.b, s);
        m->pending.push_back(t);
    }
    return e;
}

// Constants of the serial step: Angstrom_H = 1e-10 (mom6_types.F90:323), the
// hor_visc h_neglect = max(Angstrom_H, 1e-3) (mom6_hor_visc_serial.F90:203)
// and continuity's h_min = 2.0 * Angstrom_H with a default-real 2.0
// (mom6_continuity_serial.F90:211).
constexpr double kAngstromH = 1.0e-10;
static double step_hv_neglect() { return kAngstromH > 1.0e-3 ? kAngstromH : 1.0e-3; }
static double step_h_min() { return (double)2.0f * kAngstromH; }

// vert_visc_init as the driver calls it (rk2_serial_driver.F90:141-142,
// mom6_vert_visc_serial.F90:60-112), h_neglect = Angstrom_H (:151-152)
static VVParams step_vv_params(const mom6b_config& c)
{
    return VVParams{c.Kv, c.Kv_ml, c.Kv_extra_bbl, c.Hmix, kAngstromH,
                    1.0 / (c.Hbbl + kAngstromH)};
}

// barotropic_init / btstep: dtbt = dt / nstep, bebt = 0.2
// (mom6_barotropic_serial.F90:73-74, :194-195)
static BTParams step_bt_params(const mom6b_config& c)
{
    BTParams P;
    P.dtbt = c.dt / (double)c.bt_nsteps;
    P.dgeo_de = 1.0;
    P.trans_wt1 = 1.0 + 0.2;
    P.trans_wt2 = -0.2;
    P.inv_nstep = 1.0 / (double)c.bt_nsteps;
    P.nstep = c.bt_nsteps;
    P.first_direction = 0;
    P.extended = 0;
    P.spin_budget = c.wait_cycles > 0 ? c.wait_cycles : kBtDefaultWait;
    P.untiled = c.bt_untiled ? 1 : 0;
    return P;
}

// Grid quantities of the surrogate kernels.
static SurGrid sur_grid(const mom6b_model* m)
{
    SurGrid g;
    g.D = m->D;
    g.IareaT = m->M.IareaT;
    g.Datu = m->M.Datu;
    g.Datv = m->M.Datv;
    g.cor = m->M.CoriolisBu;
    g.depth = 4000.0;   // the flat bottom of init_ocean_grid (barotropic_init's Datu, Datv)
    const BTParams P = step_bt_params(m->cfg);
    g.dt_total = P.dtbt * (double)P.nstep;
    g.iu0 = P.extended ? m->D.is - 1 : m->D.is;
    g.iu1 = P.extended ? m->D.ie : m->D.ie - 1;
    g.jv0 = P.extended ? m->D.js - 1 : m->D.js;
    g.jv1 = P.extended ? m->D.je : m->D.je - 1;
    return g;
}

// One surrogate barotropic call: features of every compute cell from
// (eta, ubt, vbt), the network, and the FP64 eta advance from the divergence
// of the predicted substep-averaged transports.
static int surrogate_call(mom6b_model* m, const double* eta, const double* ubt,
                          const double* vbt, double* u_av, double* v_av, double* eta_out,
                          cudaStream_t s)
{
    const SurGrid g = sur_grid(m);
    const int nc = (m->D.ie - m->D.is + 1) * (m->D.je - m->D.js + 1);
    Mlp& N = *m->sur;
    CK(N.prepare_inference(nc));
    CK(timed(m, s, "surrogate", [&] {
        return launch_sur_features_all(g, BtInputs{eta, ubt, vbt}, N.d_norm, N.gacc, N.Xi, N.ampi, s); }));
    CK(timed(m, s, "surrogate", [&] { return N.predict(nc, s); }));
    m->launches += 1;   // predict is two launches
    CK(timed(m, s, "surrogate", [&] {
        return launch_sur_advance(g, N.outi, N.d_norm, N.ampi, eta, eta_out, u_av, v_av, s); }));
    return MOM6B_OK;
}

static int enqueue_surrogate_chain(mom6b_model* m, cudaStream_t s)
{
    const Dims& D = m->D;
    const bool fill = m->cfg.bc_fill != 0;
    if (int rc = surrogate_call(m, m->eta, m->ubt, m->vbt, m->ubt_av, m->vbt_av, m->eta_av, s))
        return rc;
    if (fill) {
        CK(timed(m, s, "halo_fill", [&] {
            return launch_halo_fill3(D, m->eta_av, m->ubt_av, m->vbt_av, 1, s); }));
    }
    if (int rc = surrogate_call(m, m->eta_av, m->ubt_av, m->vbt_av, m->ubt_av, m->vbt_av,
                                m->eta, s))
        return rc;
    if (fill)
        CK(timed(m, s, "halo_fill", [&] { return launch_halo_fill(D, m->eta, 1, 0, s); }));
    return MOM6B_OK;
}

// The plain barotropic chain from the model's (eta, ubt, vbt) into the
// shadow buffers (the check of the surrogate).
static int enqueue_shadow_chain(mom6b_model* m, cudaStream_t s)
{
    const Dims& D = m->D;
    const BTParams P = step_bt_params(m->cfg);
    CK(launch_btstep(D, m->M, m->U, m->bt, P, m->eta, m->ubt, m->vbt, m->sh_ubt_av,
                     m->sh_vbt_av, m->sh_eta_av, s));
    if (m->cfg.bc_fill) {
        CK(launch_halo_fill(D, m->sh_eta_av, 1, 0, s));
        CK(launch_halo_fill(D, m->sh_ubt_av, 1, 1, s));
        CK(launch_halo_fill(D, m->sh_vbt_av, 1, 2, s));
    }
    CK(launch_btstep(D, m->M, m->U, m->bt, P, m->sh_eta_av, m->sh_ubt_av, m->sh_vbt_av,
                     m->sh_ubt_av, m->sh_vbt_av, m->sh_eta, s));
    if (m->cfg.bc_fill) CK(launch_halo_fill(D, m->sh_eta, 1, 0, s));
    return MOM6B_OK;
}

// The FP64 continuity of one half step: zonal from hin into O.h or, with the
// meridional pass, zonal into hZ (a copy of hin, halo filled when bc_fill)
// and meridional from hZ into O.h.
static cudaError_t continuity_pass(mom6b_model* m, cudaStream_t s, const double* u,
                                   const double* v, const double* hin, const ContOut& O,
                                   double dt)
{
    const Dims& D = m->D;
    const double h_min = step_h_min();
    const double* vr_u = m->remnant ? m->visc_rem_u : nullptr;
    const double* vr_v = m->remnant ? m->visc_rem_v : nullptr;
    if (!m->merid && !m->remnant && !m->cfg.exact && continuity_fast_fits(D))
        return timed(m, s, "continuity", [&] {
            return launch_continuity_fast(D, m->M, u, hin, m->uhbt0, O, dt, h_min,
                                          m->bt.status, s); });
    if (!m->merid)
        return timed(m, s, "continuity", [&] {
            return launch_continuity(D, m->M, u, hin, m->hW, m->hE, m->uhbt0, O, m->uh_ovl,
                                     dt, h_min, s, vr_u); });
    ContOut OZ = O;
    OZ.h = m->hZ;
    cudaError_t e = cudaMemcpyAsync(m->hZ, hin, (size_t)D.plane * D.nk * sizeof(double),
                                    cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
    e = timed(m, s, "continuity", [&] {
        return launch_continuity(D, m->M, u, hin, m->hW, m->hE, m->uhbt0, OZ, m->uh_ovl, dt,
                                 h_min, s, vr_u); });
    if (e != cudaSuccess) return e;
    if (m->cfg.bc_fill) {
        e = timed(m, s, "halo_fill", [&] { return launch_halo_fill(D, m->hZ, D.nk, 0, s); });
        if (e != cudaSuccess) return e;
    }
    ContOut OV{O.h, m->vh, m->h_v, m->FA_v_S0, m->FA_v_SS, m->FA_v_N0, m->FA_v_NN,
               m->vBT_SS, m->vBT_NN, m->dv_cor};
    return timed(m, s, "continuity", [&] {
        return launch_continuity_y(D, m->M, v, m->hZ, m->hW, m->hE, m->uhbt0, OV, m->vh_ovl, dt,
                                   h_min, s, vr_v); });
}

static int enqueue_step(mom6b_model* m)
{
    const Dims& D = m->D;
    const Metrics& M = m->M;
    const mom6b_config& c = m->cfg;
    const HostGrid& g = *m->grid;
    cudaStream_t s = m->s3d;
    // The barotropic chain only needs co-residency of its own blocks; it is
    // overlapped with the 3-D chain only when enabled.
    cudaStream_t s2 = ((m->overlap_bt || m->split_bt) && !m->xfn) ? m->s2d : m->s3d;
    const double dt = c.dt;
    // the halo exchange of a decomposed run (none for a whole domain)
    auto xch = [&](double* f, int nz, int kind, int more, cudaStream_t st) -> int {
        if (!m->xfn) return MOM6B_OK;
        if (m->xfn(m->xctx, f, nz, kind, more, (void*)st) != 0)
            return fail(MOM6B_ERR_STATE, "halo exchange failed");
        return MOM6B_OK;
    };
#define XCH(f, nz, kind, more, st) \
    do { if (int rc_ = xch(f, nz, kind, more, st)) return rc_; } while (0)
    const double hv_neglect = step_hv_neglect();
    const double h_min = step_h_min();
    VVParams VV = step_vv_params(c);
    ContOut OB{m->hB, m->uh, m->h_u, m->FA_u_W0, m->FA_u_WW, m->FA_u_E0,
               m->FA_u_EE, m->uBT_WW, m->uBT_EE, m->du_cor};
    ContOut OA = OB;
    OA.h = m->hA;

    // fork the barotropic chain onto its own stream (split_bt: the caller did)
    if (s2 != s && !m->split_bt) {
        CK(cudaEventRecord(m->ev_fork, s));
        CK(cudaStreamWaitEvent(s2, m->ev_fork, 0));
    }

    if (c.precision == MOM6B_MIXED) {
        auto F = [](double* p) { return (float*)p; };
        const float hvn = (float)hv_neglect;
        // ---- predictor ----
        CK(timed(m, s, "tendency", [&] {
            return launch_tendency_f(D, M, m->U, F(m->u), F(m->v), F(m->h0), F(m->u), F(m->v),
                                     F(m->up), F(m->vp), (float)dt, hvn, s); }));
        CK(timed(m, s, "vertvisc", [&] {
            if (c.mixed_f32_vertvisc || !vertvisc_fast_fits(D))
                return launch_vertvisc_f(D, M, F(m->up), F(m->vp), F(m->h0), dt, VV, m->taux_bot,
                                         m->tauy_bot, s, c.mixed_f32_vertvisc != 0);
            return launch_vertvisc_fast_f(D, M, F(m->up), F(m->vp), F(m->h0), dt, VV,
                                          m->taux_bot, m->tauy_bot, s); }));
        CK(timed(m, s, "continuity", [&] {
            return launch_continuity_f(D, M, F(m->up), F(m->h0), F(m->hW), F(m->hE), m->uhbt0,
                                       F(m->hB), F(m->uh), F(m->h_u), OB, m->uh_ovl, dt, h_min,
                                       s); }));
        if (c.bc_fill) {
            CK(timed(m, s, "halo_fill", [&] {
                return launch_halo_fill3_f(D, F(m->hB), F(m->up), F(m->vp), g.nk, s); }));
        }
        // ---- corrector ----
        CK(timed(m, s, "tendency", [&] {
            return launch_tendency_f(D, M, m->U, F(m->up), F(m->vp), F(m->hB), F(m->u), F(m->v),
                                     F(m->u), F(m->v), (float)(0.5 * dt), hvn, s); }));
        CK(timed(m, s, "vertvisc", [&] {
            if (c.mixed_f32_vertvisc || !vertvisc_fast_fits(D))
                return launch_vertvisc_f(D, M, F(m->u), F(m->v), F(m->hB), 0.5 * dt, VV,
                                         m->taux_bot, m->tauy_bot, s,
                                         c.mixed_f32_vertvisc != 0);
            return launch_vertvisc_fast_f(D, M, F(m->u), F(m->v), F(m->hB), 0.5 * dt, VV,
                                          m->taux_bot, m->tauy_bot, s); }));
        CK(timed(m, s, "continuity", [&] {
            return launch_continuity_f(D, M, F(m->u), F(m->hB), F(m->hW), F(m->hE), m->uhbt0,
                                       F(m->hA), F(m->uh), F(m->h_u), OA, m->uh_ovl, 0.5 * dt,
                                       h_min, s); }));
        if (c.bc_fill) {
            CK(timed(m, s, "halo_fill", [&] {
                return launch_halo_fill3_f(D, F(m->hA), F(m->u), F(m->v), g.nk, s); }));
        }
    } else {
    // ---- predictor ----  (with the driver's diagnostics, diffu and diffv are kept)
    if (m->hvgen) {
        // the general hor_visc, then the tendency on its accelerations (the
        // predictor's are the driver diagnostics' diffu, diffv)
        double* du = m->diag_driver ? m->dg_du : m->hv_du;
        double* dv = m->diag_driver ? m->dg_dv : m->hv_dv;
        CK(timed(m, s, "hor_visc", [&] {
            return launch_hor_visc_gen(D, M, m->U, m->hvp, m->u, m->v, m->h0, du, dv, s); }));
        CK(timed(m, s, "tendency", [&] {
            return launch_tendency(D, M, m->U, m->u, m->v, m->h0, m->u, m->v, m->up, m->vp, dt,
                                   hv_neglect, s, du, dv, m->cor_scheme, true); }));
    } else {
    const bool td_fast = !c.exact && !m->diag_driver && m->cor_scheme == 1;
    CK(timed(m, s, "tendency", [&] {
        if (td_fast)
            return launch_tendency_fast(D, M, m->U, m->u, m->v, m->h0, m->u, m->v, m->up, m->vp,
                                        dt, hv_neglect, s, m->bt.status);
        return launch_tendency(D, M, m->U, m->u, m->v, m->h0, m->u, m->v, m->up, m->vp, dt,
                               hv_neglect, s, m->diag_driver ? m->dg_du : nullptr,
                               m->diag_driver ? m->dg_dv : nullptr, m->cor_scheme, false,
                               m->bt.status); }));
    }
    const bool vv_fast = !c.exact && !m->remnant && vertvisc_fast_fits(D);
    CK(timed(m, s, "vertvisc", [&] {
        if (vv_fast)
            return launch_vertvisc_fast(D, M, m->up, m->vp, m->h0, dt, VV, m->taux_bot,
                                        m->tauy_bot, s);
        return launch_vertvisc(D, M, m->up, m->vp, m->h0, dt, VV, m->taux_bot,
                               m->tauy_bot, s, m->remnant ? m->visc_rem_u : nullptr,
                               m->remnant ? m->visc_rem_v : nullptr); }));
    XCH(m->up, g.nk, 1, 1, s);   // rk2_mpi_cuda_c_driver.F90:409-412
    XCH(m->vp, g.nk, 2, 0, s);
    CK(continuity_pass(m, s, m->up, m->vp, m->h0, OB, dt));
    XCH(m->hB, g.nk, 0, 0, s);
    if (c.bc_fill) {
        CK(timed(m, s, "halo_fill", [&] {
            return launch_halo_fill3(D, m->hB, m->up, m->vp, g.nk, s); }));
    }
    // ---- corrector ----
    if (m->hvgen) {
        CK(timed(m, s, "hor_visc", [&] {
            return launch_hor_visc_gen(D, M, m->U, m->hvp, m->up, m->vp, m->hB, m->hv_du,
                                       m->hv_dv, s); }));
        CK(timed(m, s, "tendency", [&] {
            return launch_tendency(D, M, m->U, m->up, m->vp, m->hB, m->u, m->v, m->u, m->v,
                                   0.5 * dt, hv_neglect, s, m->hv_du, m->hv_dv, m->cor_scheme,
                                   true); }));
    } else {
    const bool td_fast = !c.exact && m->cor_scheme == 1;
    CK(timed(m, s, "tendency", [&] {
        if (td_fast)
            return launch_tendency_fast(D, M, m->U, m->up, m->vp, m->hB, m->u, m->v, m->u, m->v,
                                        0.5 * dt, hv_neglect, s, m->bt.status);
        return launch_tendency(D, M, m->U, m->up, m->vp, m->hB, m->u, m->v, m->u, m->v,
                               0.5 * dt, hv_neglect, s, nullptr, nullptr, m->cor_scheme, false,
                               m->bt.status); }));
    }
    CK(timed(m, s, "vertvisc", [&] {
        if (vv_fast)
            return launch_vertvisc_fast(D, M, m->u, m->v, m->hB, 0.5 * dt, VV, m->taux_bot,
                                        m->tauy_bot, s);
        return launch_vertvisc(D, M, m->u, m->v, m->hB, 0.5 * dt, VV, m->taux_bot,
                               m->tauy_bot, s, m->remnant ? m->visc_rem_u : nullptr,
                               m->remnant ? m->visc_rem_v : nullptr); }));
    XCH(m->u, g.nk, 1, 1, s);
    XCH(m->v, g.nk, 2, 0, s);
    CK(continuity_pass(m, s, m->u, m->v, m->hB, OA, 0.5 * dt));
    if (c.bc_fill) {
        CK(timed(m, s, "halo_fill", [&] {
            return launch_halo_fill3(D, m->hA, m->u, m->v, g.nk, s); }));
    }

    }

    // ---- barotropic chain ----
    if (m->sur && m->sur_on && !m->sur_fallen) {
        int rc = enqueue_surrogate_chain(m, s2);
        if (rc) return rc;
        if (s2 != s) {
            CK(cudaEventRecord(m->ev_join, s2));
            CK(cudaStreamWaitEvent(s, m->ev_join, 0));
        }
        return MOM6B_OK;
    }
    BTParams P = step_bt_params(c);
    P.stall_test = m->stall_test;
    if (m->xfn) {
        // a subdomain: one launch per substep, the eta, ubt, vbt halos
        // exchanged before each (rk2_mpi_cuda_c_driver.F90:376-401)
        auto bt_sub = [&](const double* ei, const double* ui, const double* vi, double* ua,
                          double* va, double* ea) -> int {
            BTParams Q = P;
            Q.substep = kBtInit;
            CK(timed(m, s2, "btstep", [&] {
                return launch_btstep(D, M, m->U, m->bt, Q, ei, ui, vi, ua, va, ea, s2); }));
            for (int n = 1; n <= P.nstep; ++n) {
                XCH(m->bt.ubt, 1, 1, 1, s2);
                XCH(m->bt.vbt, 1, 2, 1, s2);
                XCH(m->bt.eta, 1, 0, 0, s2);
                Q.substep = n;
                CK(timed(m, s2, "btstep", [&] {
                    return launch_btstep(D, M, m->U, m->bt, Q, ei, ui, vi, ua, va, ea, s2); }));
            }
            Q.substep = kBtFinish;
            CK(timed(m, s2, "btstep", [&] {
                return launch_btstep(D, M, m->U, m->bt, Q, ei, ui, vi, ua, va, ea, s2); }));
            return MOM6B_OK;
        };
        if (int rc = bt_sub(m->eta, m->ubt, m->vbt, m->ubt_av, m->vbt_av, m->eta_av)) return rc;
        return bt_sub(m->eta_av, m->ubt_av, m->vbt_av, m->ubt_av, m->vbt_av, m->eta);
    }
#undef XCH
    CK(timed(m, s2, "btstep", [&] {
        return launch_btstep(D, M, m->U, m->bt, P, m->eta, m->ubt, m->vbt, m->ubt_av,
                             m->vbt_av, m->eta_av, s2); }));
    if (c.bc_fill) {
        CK(timed(m, s2, "halo_fill", [&] {
            return launch_halo_fill3(D, m->eta_av, m->ubt_av, m->vbt_av, 1, s2); }));
    }
    CK(timed(m, s2, "btstep", [&] {
        return launch_btstep(D, M, m->U, m->bt, P, m->eta_av, m->ubt_av, m->vbt_av,
                             m->ubt_av, m->vbt_av, m->eta, s2); }));
    if (c.bc_fill)
        CK(timed(m, s2, "halo_fill", [&] { return launch_halo_fill(D, m->eta, 1, 0, s2); }));
    if (s2 != s) {
        CK(cudaEventRecord(m->ev_join, s2));
        CK(cudaStreamWaitEvent(s, m->ev_join, 0));
    }
    return MOM6B_OK;
}

// Capture one whole step (every kernel of both chains) into a CUDA graph.
static int capture_step(mom6b_model* m)
{
    cudaStream_t s = m->s3d;
    int64_t before = m->launches;
    bool timing = m->timing;
    m->timing = false;  // no event records inside the graph
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_step(m);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    m->timing = timing;
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(MOM6B_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
    m->graph = g;
    CK(cudaGraphInstantiate(&m->graph_exec, g, 0));
    m->launches_per_step = m->launches - before;
    m->launches = before;
    return MOM6B_OK;
}

static void invalidate_graph(mom6b_model* m)
{
    if (m->graph_exec) { cudaGraphExecDestroy(m->graph_exec); m->graph_exec = nullptr; }
    if (m->graph) { cudaGraphDestroy(m->graph); m->graph = nullptr; }
}

static int check_status(mom6b_model* m);
static int step_plain_or_graph(mom6b_model* m, int nsteps);

// One step with the shadow check: the plain barotropic chain runs into the
// shadow buffers from the same (eta, ubt, vbt), the step runs with the
// surrogate, and the relative L2 difference of the two etas over the compute
// domain decides: above the threshold the plain results replace the
// surrogate's and the model keeps the plain btstep from then on.
static int shadow_step(mom6b_model* m)
{
    cudaStream_t s = m->s3d;
    if (int rc = enqueue_shadow_chain(m, s)) return rc;
    if (int rc = enqueue_step(m)) return rc;
    CK(launch_sur_diff(m->D, m->eta, m->sh_eta, m->sur_acc, s));
    double acc[2] = {0.0, 0.0};
    CK(cudaMemcpyAsync(acc, m->sur_acc, sizeof(acc), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (int rc = check_status(m)) return rc;
    const double err = acc[1] > 0.0 ? std::sqrt(acc[0] / acc[1]) : std::sqrt(acc[0]);
    m->sur_last_err = err;
    m->sur_max_err = std::max(m->sur_max_err, err);
    ++m->sur_checks;
    if (!(err <= m->sur_thresh)) {
        const size_t b = m->grid->plane * sizeof(double);
        CK(cudaMemcpyAsync(m->eta, m->sh_eta, b, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(m->eta_av, m->sh_eta_av, b, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(m->ubt_av, m->sh_ubt_av, b, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(m->vbt_av, m->sh_vbt_av, b, cudaMemcpyDeviceToDevice, s));
        m->sur_fallen = true;
        ++m->sur_fallbacks;
        invalidate_graph(m);
    }
    return MOM6B_OK;
}

// Steps with the driver's diagnostics (rk2_serial_driver.F90:299-304 and
// :385-391): after every iteration the product sums of the predictor's diffu,
// diffv with the predicted thickness hB (neither changes in the corrector, so
// posting them after the whole iteration posts what the driver posts after
// the predictor's continuity), after the last iteration KE and mass.
static int diag_driver_steps(mom6b_model* m, int nsteps)
{
    cudaStream_t s = m->s3d;
    DiagCtrl& G = *m->diag;
    for (int n = 0; n < nsteps; ++n) {
        if (int rc = enqueue_step(m)) return rc;
        if (G.post_product_sum(m->id_diffu_sum, m->dg_du, m->hB, true, s) ||
            G.post_product_sum(m->id_diffv_sum, m->dg_dv, m->hB, false, s))
            return fail(MOM6B_ERR_CUDA, "diagnostic post failed");
        if (int rc = check_status(m)) return rc;
    }
    if (nsteps > 0 && (m->id_KE > 0 || m->id_mass > 0)) {
        if (m->id_KE > 0) {
            CK(launch_diag_KE(m->D, m->u, m->v, m->dg_ke, s));
            if (G.post_3d(m->id_KE, m->dg_ke, s)) return fail(MOM6B_ERR_CUDA, "diagnostic post failed");
        }
        if (m->id_mass > 0) {
            CK(launch_diag_mass(m->D, m->hA, m->dg_mass, s));
            if (G.post_2d(m->id_mass, m->dg_mass, s)) return fail(MOM6B_ERR_CUDA, "diagnostic post failed");
        }
    }
    return MOM6B_OK;
}

extern "C" int mom6b_step(mom6b_model* m, int nsteps)
{
    if (!m || nsteps < 0) return fail(MOM6B_ERR_ARG, "bad argument");
    CK(cudaSetDevice(m->cfg.device));
    if (m->cfg.cuts && !m->xfn)
        return fail(MOM6B_ERR_STATE, "a subdomain with cuts needs a halo exchange");
    if (m->xfn && (m->diag_driver || m->diag || m->merid || m->remnant || m->hvgen ||
                   m->cor_scheme != 1 || (m->sur && m->sur_on)))
        return fail(MOM6B_ERR_STATE, "the decomposed step supports the default FP64 step only");
    if (m->diag_driver) return diag_driver_steps(m, nsteps);
    if (m->sur && m->sur_on && !m->sur_fallen) {
        for (int n = 0; n < nsteps; ++n) {
            const bool shadow = m->sur_every > 0 && (m->sur_steps % m->sur_every) == 0 &&
                                !m->sur_fallen;
            ++m->sur_steps;
            if (shadow) {
                if (int rc = shadow_step(m)) return rc;
                continue;
            }
            if (int rc = step_plain_or_graph(m, 1)) return rc;
        }
        return MOM6B_OK;
    }
    return step_plain_or_graph(m, nsteps);
}

static int step_plain_or_graph(mom6b_model* m, int nsteps)
{
    if (m->cfg.use_graph && !m->timing && !m->xfn) {
        if (!m->graph_exec) {
            if (int rc = capture_step(m)) return rc;
        }
        for (int n = 0; n < nsteps; ++n) {
            CK(cudaGraphLaunch(m->graph_exec, m->s3d));
            m->launches += m->launches_per_step;
        }
        return MOM6B_OK;
    }
    for (int n = 0; n < nsteps; ++n) {
        int rc = enqueue_step(m);
        if (rc) return rc;
    }
    return MOM6B_OK;
}

static int check_status(mom6b_model* m)
{
    int st = 0;
    CK(cudaMemcpy(&st, m->bt.status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st != kDevOk) {
        cudaMemset(m->bt.status, 0, sizeof(int));
        cudaMemset(m->bt.bar_count, 0, sizeof(unsigned int));
        return fail(MOM6B_ERR_TIMEOUT, "barotropic grid barrier timed out");
    }
    return MOM6B_OK;
}

extern "C" int mom6b_synchronize(mom6b_model* m)
{
    if (!m) return fail(MOM6B_ERR_ARG, "null model");
    CK(cudaStreamSynchronize(m->s3d));
    CK(cudaStreamSynchronize(m->s2d));
    return check_status(m);
}

static double* field_ptr(mom6b_model* m, int f, bool* is3d, bool* writable)
{
    *is3d = true;
    *writable = true;
    switch (f) {
    case MOM6B_F_U: return m->u;
    case MOM6B_F_V: return m->v;
    case MOM6B_F_H: return m->hA;
    case MOM6B_F_H0: return m->h0;
    case MOM6B_F_UH: return m->uh;
    case MOM6B_F_UP: return m->up;
    case MOM6B_F_VP: return m->vp;
    case MOM6B_F_HU_BT: return m->h_u;
    case MOM6B_F_RAY_U: return m->Ray_u;
    case MOM6B_F_RAY_V: return m->Ray_v;
    case MOM6B_F_VH: return m->vh;
    case MOM6B_F_HV_BT: return m->h_v;
    case MOM6B_F_VISC_REM_U: return m->visc_rem_u;
    case MOM6B_F_VISC_REM_V: return m->visc_rem_v;
    default: break;
    }
    *is3d = false;
    switch (f) {
    case MOM6B_F_ETA: return m->eta;
    case MOM6B_F_UBT: return m->ubt;
    case MOM6B_F_VBT: return m->vbt;
    case MOM6B_F_UBT_AV: return m->ubt_av;
    case MOM6B_F_VBT_AV: return m->vbt_av;
    case MOM6B_F_ETA_AV: return m->eta_av;
    case MOM6B_F_FA_U_W0: return m->FA_u_W0;
    case MOM6B_F_FA_U_WW: return m->FA_u_WW;
    case MOM6B_F_FA_U_E0: return m->FA_u_E0;
    case MOM6B_F_FA_U_EE: return m->FA_u_EE;
    case MOM6B_F_UBT_WW: return m->uBT_WW;
    case MOM6B_F_UBT_EE: return m->uBT_EE;
    case MOM6B_F_DU_COR: return m->du_cor;
    case MOM6B_F_TAUX_BOT: return m->taux_bot;
    case MOM6B_F_TAUY_BOT: return m->tauy_bot;
    case MOM6B_F_TAUX: return m->taux;
    case MOM6B_F_TAUY: return m->tauy;
    case MOM6B_F_FA_V_S0: return m->FA_v_S0;
    case MOM6B_F_FA_V_SS: return m->FA_v_SS;
    case MOM6B_F_FA_V_N0: return m->FA_v_N0;
    case MOM6B_F_FA_V_NN: return m->FA_v_NN;
    case MOM6B_F_VBT_SS: return m->vBT_SS;
    case MOM6B_F_VBT_NN: return m->vBT_NN;
    case MOM6B_F_DV_COR: return m->dv_cor;
    default: return nullptr;
    }
}

// In the mixed form these 3-D fields are stored as FP32 in their buffers.
static bool is_f32(const mom6b_model* m, int f)
{
    if (m->cfg.precision != MOM6B_MIXED) return false;
    switch (f) {
    case MOM6B_F_U: case MOM6B_F_V: case MOM6B_F_H: case MOM6B_F_H0: case MOM6B_F_UH:
    case MOM6B_F_UP: case MOM6B_F_VP: case MOM6B_F_HU_BT: return true;
    default: return false;
    }
}

extern "C" size_t mom6b_field_size(const mom6b_model* m, int f)
{
    if (!m) return 0;
    bool is3d, w;
    if (!field_ptr(const_cast<mom6b_model*>(m), f, &is3d, &w)) return 0;
    return m->grid->plane * (is3d ? (size_t)m->grid->nk : 1);
}

extern "C" int mom6b_get_field(mom6b_model* m, int f, double* host, size_t count)
{
    if (!m || !host) return fail(MOM6B_ERR_ARG, "null argument");
    bool is3d, w;
    double* p = field_ptr(m, f, &is3d, &w);
    if (!p) return fail(MOM6B_ERR_ARG, "unknown field id");
    size_t n = mom6b_field_size(m, f);
    if (count != n) return fail(MOM6B_ERR_ARG, "count does not match the field size");
    CK(cudaSetDevice(m->cfg.device));
    CK(cudaStreamSynchronize(m->s3d));
    CK(cudaStreamSynchronize(m->s2d));
    if (is_f32(m, f)) {
        std::vector<float> tmp(n);
        CK(cudaMemcpy(tmp.data(), p, n * sizeof(float), cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < n; ++q) host[q] = (double)tmp[q];
    } else {
        CK(cudaMemcpy(host, p, n * sizeof(double), cudaMemcpyDeviceToHost));
    }
    return check_status(m);
}

extern "C" int mom6b_set_field(mom6b_model* m, int f, const double* host, size_t count)
{
    if (!m || !host) return fail(MOM6B_ERR_ARG, "null argument");
    bool is3d, w;
    double* p = field_ptr(m, f, &is3d, &w);
    if (!p || !w) return fail(MOM6B_ERR_ARG, "unknown or read-only field id");
    size_t n = mom6b_field_size(m, f);
    if (count != n) return fail(MOM6B_ERR_ARG, "count does not match the field size");
    CK(cudaSetDevice(m->cfg.device));
    CK(cudaStreamSynchronize(m->s3d));
    CK(cudaStreamSynchronize(m->s2d));
    const void* src = host;
    size_t bytes = n * sizeof(double);
    std::vector<float> tmp;
    if (is_f32(m, f)) {
        tmp.assign(host, host + n);
        src = tmp.data();
        bytes = n * sizeof(float);
    }
    CK(cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice));
    if (f == MOM6B_F_H0) {  // the step resets h to h0, halo ring included
        CK(cudaMemcpy(m->hA, src, bytes, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(m->hB, src, bytes, cudaMemcpyHostToDevice));
    }
    if (f == MOM6B_F_RAY_U || f == MOM6B_F_RAY_V) {
        std::vector<double> Ru(n), Rv(n);
        CK(cudaMemcpy(Ru.data(), m->Ray_u, n * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(Rv.data(), m->Ray_v, n * sizeof(double), cudaMemcpyDeviceToHost));
        if (int rc = set_ray_flags(m, Ru, Rv)) return rc;
    }
    return MOM6B_OK;
}

extern "C" int mom6b_field_device_ptr(mom6b_model* m, int f, void** dptr)
{
    if (!m || !dptr) return fail(MOM6B_ERR_ARG, "null argument");
    bool is3d, w;
    double* p = field_ptr(m, f, &is3d, &w);
    if (!p) return fail(MOM6B_ERR_ARG, "unknown field id");
    *dptr = p;
    return MOM6B_OK;
}

extern "C" int mom6b_metric_device_ptr(mom6b_model* m, const char* name, void** dptr)
{
    if (!m || !name || !dptr) return fail(MOM6B_ERR_ARG, "null argument");
    const Metrics& M = m->M;
    const std::map<std::string, const double*> t = {
        {"IareaT", M.IareaT}, {"IdxCu", M.IdxCu}, {"IdyCv", M.IdyCv}, {"Datu", M.Datu},
        {"Datv", M.Datv}, {"gtot_E", M.gtot_E}, {"gtot_W", M.gtot_W},
        {"gtot_N", M.gtot_N}, {"gtot_S", M.gtot_S}, {"f_4_u", M.f_4_u},
        {"f_4_v", M.f_4_v}, {"bt_rem_u", M.bt_rem_u}, {"bt_rem_v", M.bt_rem_v}};
    auto it = t.find(name);
    if (it == t.end()) return fail(MOM6B_ERR_ARG, std::string("unknown metric ") + name);
    *dptr = (void*)it->second;
    return MOM6B_OK;
}

extern "C" int mom6b_dims(const mom6b_model* m, int* o)
{
    if (!m || !o) return fail(MOM6B_ERR_ARG, "null argument");
    const HostGrid& g = *m->grid;
    o[0] = g.n1; o[1] = g.n2; o[2] = g.nk; o[3] = g.is; o[4] = g.ie; o[5] = g.js;
    o[6] = g.je; o[7] = m->cfg.bt_nsteps;
    return MOM6B_OK;
}

extern "C" int mom6b_stream(mom6b_model* m, void** stream)
{
    if (!m || !stream) return fail(MOM6B_ERR_ARG, "null argument");
    *stream = (void*)m->s3d;
    return MOM6B_OK;
}

extern "C" int mom6b_step_host(mom6b_model* m, int nsteps, double* u, double* v,
                               double* h, double* eta)
{
    if (!m || nsteps < 0) return fail(MOM6B_ERR_ARG, "bad argument");
    CK(cudaSetDevice(m->cfg.device));
    const size_t n3 = m->grid->plane * (size_t)m->grid->nk, n2 = m->grid->plane;
    cudaStream_t s = m->s3d;
    if (m->cfg.precision == MOM6B_MIXED) {  // FP32 state: convert through set/get
        if (u) if (int rc = mom6b_set_field(m, MOM6B_F_U, u, n3)) return rc;
        if (v) if (int rc = mom6b_set_field(m, MOM6B_F_V, v, n3)) return rc;
        if (h) if (int rc = mom6b_set_field(m, MOM6B_F_H, h, n3)) return rc;
        if (eta) if (int rc = mom6b_set_field(m, MOM6B_F_ETA, eta, n2)) return rc;
        if (int rc = mom6b_step(m, nsteps)) return rc;
        if (u) if (int rc = mom6b_get_field(m, MOM6B_F_U, u, n3)) return rc;
        if (v) if (int rc = mom6b_get_field(m, MOM6B_F_V, v, n3)) return rc;
        if (h) if (int rc = mom6b_get_field(m, MOM6B_F_H, h, n3)) return rc;
        if (eta) if (int rc = mom6b_get_field(m, MOM6B_F_ETA, eta, n2)) return rc;
        return check_status(m);
    }
    CK(cudaStreamSynchronize(m->s2d));
    if (u) CK(cudaMemcpyAsync(m->u, u, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
    if (v) CK(cudaMemcpyAsync(m->v, v, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
    if (h) CK(cudaMemcpyAsync(m->hA, h, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
    if (eta) CK(cudaMemcpyAsync(m->eta, eta, n2 * sizeof(double), cudaMemcpyHostToDevice, s));
    if (int rc = mom6b_step(m, nsteps)) return rc;
    if (u) CK(cudaMemcpyAsync(u, m->u, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (v) CK(cudaMemcpyAsync(v, m->v, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (h) CK(cudaMemcpyAsync(h, m->hA, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (eta) CK(cudaMemcpyAsync(eta, m->eta, n2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return check_status(m);
}

extern "C" int mom6b_step_host_io(mom6b_model* m, int nsteps, const double* u_in,
                                  const double* v_in, const double* eta_in, double* u_out,
                                  double* v_out, double* h_out, double* eta_out)
{
    if (!m || nsteps < 0) return fail(MOM6B_ERR_ARG, "bad argument");
    CK(cudaSetDevice(m->cfg.device));
    const size_t n3 = m->grid->plane * (size_t)m->grid->nk, n2 = m->grid->plane;
    cudaStream_t s = m->s3d;
    if (m->cfg.precision == MOM6B_MIXED) {  // FP32 state: convert through set/get
        if (u_in) if (int rc = mom6b_set_field(m, MOM6B_F_U, u_in, n3)) return rc;
        if (v_in) if (int rc = mom6b_set_field(m, MOM6B_F_V, v_in, n3)) return rc;
        if (eta_in) if (int rc = mom6b_set_field(m, MOM6B_F_ETA, eta_in, n2)) return rc;
        if (int rc = mom6b_step(m, nsteps)) return rc;
        if (u_out) if (int rc = mom6b_get_field(m, MOM6B_F_U, u_out, n3)) return rc;
        if (v_out) if (int rc = mom6b_get_field(m, MOM6B_F_V, v_out, n3)) return rc;
        if (h_out) if (int rc = mom6b_get_field(m, MOM6B_F_H, h_out, n3)) return rc;
        if (eta_out) if (int rc = mom6b_get_field(m, MOM6B_F_ETA, eta_out, n2)) return rc;
        return check_status(m);
    }
    CK(cudaStreamSynchronize(m->s2d));
    // One plain step: the barotropic chain reads only eta, ubt and vbt, so it
    // runs on its own stream as soon as eta has arrived, while u and v are
    // still being uploaded for the 3-D chain (eager launches; the fields equal
    // those of mom6b_step).
    const bool split = nsteps == 1 && !m->cfg.cuts && !m->xfn && !m->diag_driver &&
                       !(m->sur && m->sur_on) && !m->timing;
    if (split) {
        CK(cudaEventRecord(m->ev_fork, s));
        CK(cudaStreamWaitEvent(m->s2d, m->ev_fork, 0));
        if (eta_in)
            CK(cudaMemcpyAsync(m->eta, eta_in, n2 * sizeof(double), cudaMemcpyHostToDevice,
                               m->s2d));
    }
    if (u_in) CK(cudaMemcpyAsync(m->u, u_in, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
    if (v_in) CK(cudaMemcpyAsync(m->v, v_in, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
    if (split) {
        m->split_bt = true;
        const int rc = enqueue_step(m);
        m->split_bt = false;
        if (rc) return rc;
    } else {
        if (eta_in)
            CK(cudaMemcpyAsync(m->eta, eta_in, n2 * sizeof(double), cudaMemcpyHostToDevice, s));
        if (int rc = mom6b_step(m, nsteps)) return rc;
    }
    if (u_out) CK(cudaMemcpyAsync(u_out, m->u, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (v_out) CK(cudaMemcpyAsync(v_out, m->v, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (h_out) CK(cudaMemcpyAsync(h_out, m->hA, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (eta_out)
        CK(cudaMemcpyAsync(eta_out, m->eta, n2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return check_status(m);
}

extern "C" int mom6b_verify(mom6b_model* m, double* out)
{
    if (!m || !out) return fail(MOM6B_ERR_ARG, "null argument");
    const HostGrid& g = *m->grid;
    size_t n3 = g.plane * (size_t)g.nk;
    std::vector<double> h0(n3), h(n3), u(n3), v(n3), eta(g.plane);
    if (int rc = mom6b_get_field(m, MOM6B_F_H0, h0.data(), n3)) return rc;
    if (int rc = mom6b_get_field(m, MOM6B_F_H, h.data(), n3)) return rc;
    if (int rc = mom6b_get_field(m, MOM6B_F_U, u.data(), n3)) return rc;
    if (int rc = mom6b_get_field(m, MOM6B_F_V, v.data(), n3)) return rc;
    if (int rc = mom6b_get_field(m, MOM6B_F_ETA, eta.data(), g.plane)) return rc;
    // verify_state, rk2_serial_driver.F90:563-623, summed in the same order
    double mi = 0.0, mf = 0.0, mu = 0.0, mv = 0.0, me = 0.0, ke = 0.0;
    for (int k = 1; k <= g.nk; ++k)
        for (int j = g.js; j <= g.je; ++j)
            for (int i = g.is; i <= g.ie; ++i) {
                size_t p = g.at(i, j, k);
                double a = g.areaT[g.at(i, j)];
                mi = mi + h0[p] * a;
                mf = mf + h[p] * a;
                mu = std::max(mu, std::fabs(u[p]));
                mv = std::max(mv, std::fabs(v[p]));
                ke = ke + 0.5 * (u[p] * u[p] + v[p] * v[p]) * h[p] * a;
            }
    for (int j = g.js; j <= g.je; ++j)
        for (int i = g.is; i <= g.ie; ++i) me = std::max(me, std::fabs(eta[g.at(i, j)]));
    out[0] = mi; out[1] = mf; out[2] = std::fabs(mf - mi) / mi;
    out[3] = mu; out[4] = mv; out[5] = me; out[6] = ke;
    return MOM6B_OK;
}

extern "C" int64_t mom6b_launch_count(const mom6b_model* m) { return m ? m->launches : 0; }
extern "C" void mom6b_reset_launch_count(mom6b_model* m)
{
    if (m) m->launches = 0;
}

extern "C" int mom6b_kernel_timing(mom6b_model* m, int enable)
{
    if (!m) return fail(MOM6B_ERR_ARG, "null model");
    m->timing = enable != 0;
    m->timed.clear();
    return MOM6B_OK;
}

extern "C" int mom6b_kernel_time_ms(mom6b_model* m, const char* kernel, double* avg_ms,
                                    int64_t* launches)
{
    if (!m || !kernel) return fail(MOM6B_ERR_ARG, "null argument");
    CK(cudaStreamSynchronize(m->s3d));
    CK(cudaStreamSynchronize(m->s2d));
    for (auto& t : m->pending) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t.a, t.b);
        auto& e = m->timed[t.name];
        e.first += ms;
        e.second += 1;
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    m->pending.clear();
    auto it = m->timed.find(kernel);
    if (it == m->timed.end()) {
        if (avg_ms) *avg_ms = 0.0;
        if (launches) *launches = 0;
        return MOM6B_OK;
    }
    if (avg_ms) *avg_ms = it->second.first / (double)it->second.second;
    if (launches) *launches = it->second.second;
    return MOM6B_OK;
}

// ===========================================================================
// Ensemble: many independent domains of uneven size in the mixed form, one
// launch per phase for all of them (k_ensemble.cu, k_btstep.cu).
// ===========================================================================
// Each domain is a full mixed-form model (its own allocations, initial state
// and halo fill, exactly as mom6b_create builds it); the ensemble adds the
// device table of domain descriptors, the per-phase block tables of the
// current tuning, the barotropic tile list and its flags, and a stream and
// CUDA graph of its own.  One step is fourteen launches whatever the number
// of domains (ten when no domain fills halos): tendency, vertvisc, PPM edges,
// faces and halo fill for the predictor and the corrector, then the two
// barotropic calls with their halo fills.
// ---------------------------------------------------------------------------
// diagnostics (mom6_diag.F90) and binary field dumps
// ---------------------------------------------------------------------------
static int diag_ready(mom6b_model* m)
{
    if (!m) return fail(MOM6B_ERR_ARG, "null model");
    if (!m->diag || !m->diag->initialized()) return fail(MOM6B_ERR_STATE, "diagnostics not initialized");
    CK(cudaSetDevice(m->cfg.device));
    return MOM6B_OK;
}

extern "C" int mom6b_diag_init(mom6b_model* m, const char* output_dir, int output_freq)
{
    if (!m || !output_dir) return fail(MOM6B_ERR_ARG, "null argument");
    if (output_freq < 1) return fail(MOM6B_ERR_ARG, "output_freq must be at least 1");
    CK(cudaSetDevice(m->cfg.device));
    if (m->diag && m->diag->initialized()) return MOM6B_OK;   // as diag_init: once
    m->diag.reset(new DiagCtrl());
    if (m->diag->init(m->D, output_dir, output_freq, m->s3d))
        return fail(MOM6B_ERR_NOMEM, "diagnostic work array");
    return MOM6B_OK;
}

extern "C" int mom6b_diag_end(mom6b_model* m)
{
    if (!m) return fail(MOM6B_ERR_ARG, "null model");
    CK(cudaSetDevice(m->cfg.device));
    CK(cudaStreamSynchronize(m->s3d));
    m->diag.reset();
    m->diag_driver = false;
    m->id_KE = m->id_diffu_sum = m->id_diffv_sum = m->id_mass = -1;
    return MOM6B_OK;
}

extern "C" int mom6b_diag_register(mom6b_model* m, const char* name, const char* long_name,
                                   const char* units, int ndims, const char* position,
                                   int output_mode, int* id)
{
    if (int rc = diag_ready(m)) return rc;
    if (!name || !long_name || !units || !position || !id) return fail(MOM6B_ERR_ARG, "null argument");
    if (ndims != 2 && ndims != 3) return fail(MOM6B_ERR_ARG, "ndims must be 2 or 3");
    *id = m->diag->register_field(name, long_name, units, ndims, position, output_mode);
    return MOM6B_OK;
}

static int diag_post(mom6b_model* m, int id, const double* a, const double* b, int kind)
{
    if (int rc = diag_ready(m)) return rc;
    if (id <= 0) return MOM6B_OK;   // inactive diagnostic: nothing to do
    if (!m->diag->field(id)) return fail(MOM6B_ERR_ARG, "unknown diagnostic id");
    if (!a || (kind >= 2 && !b)) return fail(MOM6B_ERR_ARG, "null field");
    int rc;
    switch (kind) {
    case 0: rc = m->diag->post_2d(id, a, m->s3d); break;
    case 1: rc = m->diag->post_3d(id, a, m->s3d); break;
    default: rc = m->diag->post_product_sum(id, a, b, kind == 2, m->s3d); break;
    }
    return rc ? fail(MOM6B_ERR_CUDA, "diagnostic post failed") : MOM6B_OK;
}

extern "C" int mom6b_diag_post_2d(mom6b_model* m, int id, const double* field)
{
    return diag_post(m, id, field, nullptr, 0);
}

extern "C" int mom6b_diag_post_3d(mom6b_model* m, int id, const double* field)
{
    return diag_post(m, id, field, nullptr, 1);
}

extern "C" int mom6b_diag_post_product_sum_u(mom6b_model* m, int id, const double* u_a,
                                             const double* u_b)
{
    return diag_post(m, id, u_a, u_b, 2);
}

extern "C" int mom6b_diag_post_product_sum_v(mom6b_model* m, int id, const double* v_a,
                                             const double* v_b)
{
    return diag_post(m, id, v_a, v_b, 3);
}

extern "C" int mom6b_diag_stats(const mom6b_model* m, int id, double* out4)
{
    if (!m || !out4) return fail(MOM6B_ERR_ARG, "null argument");
    if (!m->diag) return fail(MOM6B_ERR_STATE, "diagnostics not initialized");
    const DiagField* F = m->diag->field(id);
    if (!F) return fail(MOM6B_ERR_ARG, "unknown diagnostic id");
    if (!F->posted) return fail(MOM6B_ERR_STATE, "diagnostic not posted yet");
    for (int q = 0; q < 4; ++q) out4[q] = F->stats[q];
    return MOM6B_OK;
}

extern "C" int mom6b_diag_report(mom6b_model* m, int* out3)
{
    if (int rc = diag_ready(m)) return rc;
    std::printf("\nDiagnostic Summary:\n--------------------------------------------------\n"
                "  Registered diagnostics:  %8d\n  Total post_data calls:   %8d\n",
                m->diag->num_diags(), m->diag->total_calls());
    std::fflush(stdout);
    if (out3) {
        out3[0] = m->diag->num_diags();
        out3[1] = m->diag->total_calls();
        out3[2] = m->diag->call_count();
    }
    return MOM6B_OK;
}

extern "C" int mom6b_diag_driver(mom6b_model* m, int output_mode)
{
    if (int rc = diag_ready(m)) return rc;
    if (m->cfg.precision != MOM6B_FP64)
        return fail(MOM6B_ERR_STATE, "the driver's diagnostics need the FP64 form");
    if (m->sur && m->sur_on) return fail(MOM6B_ERR_STATE, "disable the surrogate first");
    DiagCtrl& G = *m->diag;
    m->id_KE = G.register_field("KE", "Kinetic Energy", "m2/s2", 3, "h", output_mode);
    m->id_diffu_sum = G.register_field("diffu_sum", "Vertically summed u-diffusion", "m/s2", 2,
                                       "u", output_mode);
    m->id_diffv_sum = G.register_field("diffv_sum", "Vertically summed v-diffusion", "m/s2", 2,
                                       "v", output_mode);
    m->id_mass = G.register_field("mass", "Vertically summed thickness", "m", 2, "h",
                                  output_mode);
    if (!m->dg_du) {
        cudaError_t e = cudaSuccess;
        const size_t n3 = (size_t)m->D.plane * m->D.nk, n2 = (size_t)m->D.plane;
        m->dg_du = dalloc(m, n3, &e);
        m->dg_dv = dalloc(m, n3, &e);
        m->dg_ke = dalloc(m, n3, &e);
        m->dg_mass = dalloc(m, n2, &e);
        if (e != cudaSuccess || !m->dg_du || !m->dg_dv || !m->dg_ke || !m->dg_mass)
            return fail(MOM6B_ERR_NOMEM, "diagnostic fields");
    }
    m->diag_driver = true;
    invalidate_graph(m);   // the predictor's tendency launch changes
    return MOM6B_OK;
}

extern "C" int mom6b_set_coriolis_scheme(mom6b_model* m, int scheme)
{
    if (!m || scheme < 1 || scheme > 3) return fail(MOM6B_ERR_ARG, "scheme must be 1, 2 or 3");
    if (scheme != 1 && m->cfg.precision != MOM6B_FP64)
        return fail(MOM6B_ERR_STATE, "the Arakawa schemes are built for the FP64 form");
    CK(cudaSetDevice(m->cfg.device));
    CK(cudaStreamSynchronize(m->s3d));
    m->cor_scheme = scheme;
    invalidate_graph(m);
    return MOM6B_OK;
}

extern "C" int mom6b_set_continuity_merid(mom6b_model* m, int on)
{
    if (!m) return fail(MOM6B_ERR_ARG, "null model");
    if (on && m->cfg.precision != MOM6B_FP64)
        return fail(MOM6B_ERR_STATE, "the meridional pass is built for the FP64 form");
    CK(cudaSetDevice(m->cfg.device));
    CK(cudaStreamSynchronize(m->s3d));
    if (on && !m->hZ) {
        cudaError_t e = cudaSuccess;
        const size_t n3 = (size_t)m->D.plane * m->D.nk, n2 = (size_t)m->D.plane;
        m->hZ = dalloc(m, n3, &e);
        m->vh = dalloc(m, n3, &e);
        m->h_v = dalloc(m, n3, &e);
        m->vh_ovl = dalloc(m, continuity_overlap_doubles_y(m->D), &e);
        double** two[] = {&m->FA_v_S0, &m->FA_v_SS, &m->FA_v_N0, &m->FA_v_NN,
                          &m->vBT_SS, &m->vBT_NN, &m->dv_cor};
        for (double** p : two) *p = dalloc(m, n2, &e);
        if (e != cudaSuccess) return fail(MOM6B_ERR_NOMEM, "meridional continuity buffers");
    }
    m->merid = on != 0;
    invalidate_graph(m);
    return MOM6B_OK;
}

extern "C" int mom6b_set_bt_overlap(mom6b_model* m, int on)
{
    if (!m) return fail(MOM6B_ERR_ARG, "null model");
    CK(cudaSetDevice(m->cfg.device));
    CK(cudaStreamSynchronize(m->s3d));
    CK(cudaStreamSynchronize(m->s2d));
    m->overlap_bt = on != 0;
    invalidate_graph(m);
    return MOM6B_OK;
}

extern "C" int mom6b_set_wait_limit(mom6b_model* m, long long cycles, int stall_test)
{
    if (!m || cycles < 0) return fail(MOM6B_ERR_ARG, "bad argument");
    CK(cudaSetDevice(m->cfg.device));
    CK(cudaStreamSynchronize(m->s3d));
    CK(cudaStreamSynchronize(m->s2d));
    m->cfg.wait_cycles = cycles;
    m->stall_test = stall_test ? 1 : 0;
    invalidate_graph(m);
    return MOM6B_OK;
}

extern "C" int mom6b_set_exchange(mom6b_model* m, mom6b_exchange_fn fn, void* ctx)
{
    if (!m) return fail(MOM6B_ERR_ARG, "null model");
    CK(cudaSetDevice(m->cfg.device));
    CK(cudaStreamSynchronize(m->s3d));
    CK(cudaStreamSynchronize(m->s2d));
    m->xfn = fn;
    m->xctx = fn ? ctx : nullptr;
    invalidate_graph(m);
    return MOM6B_OK;
}

// ---- the in-process halo group --------------------------------------------
// Members post their field, meet at a host barrier, pull their neighbours'
// strips with 3-D copies on their own streams (peer copies across devices),
// and meet again before any owner may change its strips.
struct mom6b_halo_group {
    int px = 0, py = 0;
    double timeout_s = 60.0;
    std::mutex mu;
    std::condition_variable cv;
    int arrived = 0;
    unsigned long long gen = 0;
    bool failed = false;
    struct Member {
        mom6b_model* m = nullptr;
        std::vector<std::pair<double*, int>> posted;   // the fields of the open point
    };
    std::vector<Member> mem;
    struct Ctx {
        mom6b_halo_group* g;
        int rank;
    };
    std::vector<std::unique_ptr<Ctx>> ctx;
    int rank_at(int x, int y) const { return (x >= 0 && x < px && y >= 0 && y < py) ? x * py + y : -1; }
};

static bool group_meet(mom6b_halo_group* g)
{
    std::unique_lock<std::mutex> lk(g->mu);
    if (g->failed) return false;
    const unsigned long long my = g->gen;
    if (++g->arrived == (int)g->mem.size()) {
        g->arrived = 0;
        ++g->gen;
        g->cv.notify_all();
        return true;
    }
    const bool met = g->cv.wait_for(lk, std::chrono::duration<double>(g->timeout_s),
                                    [&] { return g->gen != my || g->failed; });
    if (!met || g->failed) {
        g->failed = true;
        g->cv.notify_all();
        return false;
    }
    return true;
}

static int group_exchange(void* vctx, double* field, int nz, int kind, int more, void* stream)
{
    (void)kind;
    auto* c = (mom6b_halo_group::Ctx*)vctx;
    mom6b_halo_group* g = c->g;
    const int r = c->rank;
    cudaStream_t s = (cudaStream_t)stream;
    mom6b_halo_group::Member& me = g->mem[r];
    me.posted.emplace_back(field, nz);
    if (more) return 0;   // the point's other fields follow
    if (cudaStreamSynchronize(s) != cudaSuccess || !group_meet(g)) {
        std::lock_guard<std::mutex> lk(g->mu);
        g->failed = true;
        g->cv.notify_all();
        me.posted.clear();
        return 1;
    }
    const int hw = 3;
    const Dims& D = me.m->D;
    const int x = r / g->py, y = r % g->py;
    const bool hw_ = g->rank_at(x - 1, y) >= 0, he = g->rank_at(x + 1, y) >= 0;
    const bool hs = g->rank_at(x, y - 1) >= 0, hn = g->rank_at(x, y + 1) >= 0;
    const int r0 = hs ? hw : 0, r1 = hn ? D.n2 - hw : D.n2;   // east / west strip rows
    const int c0 = hw_ ? hw : 0, c1 = he ? D.n1 - hw : D.n1;  // north / south strip columns
    int bad = 0;
    for (size_t fi = 0; fi < me.posted.size() && !bad; ++fi)
    for (int dy = -1; dy <= 1 && !bad; ++dy)
        for (int dx = -1; dx <= 1 && !bad; ++dx) {
            if (!dx && !dy) continue;
            const int nr = g->rank_at(x + dx, y + dy);
            if (nr < 0) continue;
            const mom6b_halo_group::Member& nb = g->mem[nr];
            const Dims& N = nb.m->D;
            if (nb.posted.size() != me.posted.size() || nb.posted[fi].second != me.posted[fi].second) {
                bad = 1;
                break;
            }
            double* field = me.posted[fi].first;
            const int nz = me.posted[fi].second;
            const double* src = nb.posted[fi].first;
            // this member's receive box and the neighbour's send box (0-based)
            const int mx0 = dx > 0 ? D.n1 - hw : (dx < 0 ? 0 : c0);
            const int mx1 = dx > 0 ? D.n1 : (dx < 0 ? hw : c1);
            const int my0 = dy > 0 ? D.n2 - hw : (dy < 0 ? 0 : r0);
            const int my1 = dy > 0 ? D.n2 : (dy < 0 ? hw : r1);
            const int sx0 = dx > 0 ? hw : (dx < 0 ? N.n1 - 2 * hw : c0);
            const int sy0 = dy > 0 ? hw : (dy < 0 ? N.n2 - 2 * hw : r0);
            const size_t w = (size_t)(mx1 - mx0), h = (size_t)(my1 - my0);
            const int dd = me.m->cfg.device, sd = nb.m->cfg.device;
            cudaError_t e;
            if (dd == sd) {
                cudaMemcpy3DParms p = {};
                p.srcPtr = make_cudaPitchedPtr((void*)src, (size_t)N.n1 * 8, N.n1, N.n2);
                p.srcPos = make_cudaPos((size_t)sx0 * 8, sy0, 0);
                p.dstPtr = make_cudaPitchedPtr((void*)field, (size_t)D.n1 * 8, D.n1, D.n2);
                p.dstPos = make_cudaPos((size_t)mx0 * 8, my0, 0);
                p.extent = make_cudaExtent(w * 8, h, (size_t)nz);
                p.kind = cudaMemcpyDeviceToDevice;
                e = cudaMemcpy3DAsync(&p, s);
            } else {
                cudaMemcpy3DPeerParms p = {};
                p.srcPtr = make_cudaPitchedPtr((void*)src, (size_t)N.n1 * 8, N.n1, N.n2);
                p.srcPos = make_cudaPos((size_t)sx0 * 8, sy0, 0);
                p.srcDevice = sd;
                p.dstPtr = make_cudaPitchedPtr((void*)field, (size_t)D.n1 * 8, D.n1, D.n2);
                p.dstPos = make_cudaPos((size_t)mx0 * 8, my0, 0);
                p.dstDevice = dd;
                p.extent = make_cudaExtent(w * 8, h, (size_t)nz);
                e = cudaMemcpy3DPeerAsync(&p, s);
            }
            if (e != cudaSuccess) bad = 1;
        }
    if (bad || cudaStreamSynchronize(s) != cudaSuccess) {
        // the neighbours may still be reading this member's posts: they stay
        // (the group is failed, so no later round reads them)
        std::lock_guard<std::mutex> lk(g->mu);
        g->failed = true;
        g->cv.notify_all();
        return 1;
    }
    const bool ok = group_meet(g);   // no member reads the posts after this
    me.posted.clear();
    return ok ? 0 : 1;
}

extern "C" int mom6b_halo_group_create(int npes_x, int npes_y, double timeout_s,
                                       mom6b_halo_group** out)
{
    if (!out || npes_x < 1 || npes_y < 1 || npes_x * npes_y > 4096 || !(timeout_s > 0.0))
        return fail(MOM6B_ERR_ARG, "bad halo group layout");
    auto g = std::make_unique<mom6b_halo_group>();
    g->px = npes_x;
    g->py = npes_y;
    g->timeout_s = timeout_s;
    g->mem.resize((size_t)npes_x * npes_y);
    *out = g.release();
    return MOM6B_OK;
}

extern "C" int mom6b_halo_group_join(mom6b_halo_group* g, mom6b_model* m, int rank)
{
    if (!g || !m || rank < 0 || rank >= (int)g->mem.size())
        return fail(MOM6B_ERR_ARG, "bad halo group member");
    if (g->mem[rank].m) return fail(MOM6B_ERR_STATE, "rank already joined");
    const int x = rank / g->py, y = rank % g->py;
    const int want = (g->rank_at(x - 1, y) >= 0 ? MOM6B_CUT_W : 0) |
                     (g->rank_at(x + 1, y) >= 0 ? MOM6B_CUT_E : 0) |
                     (g->rank_at(x, y - 1) >= 0 ? MOM6B_CUT_S : 0) |
                     (g->rank_at(x, y + 1) >= 0 ? MOM6B_CUT_N : 0);
    if (m->cfg.cuts != want) return fail(MOM6B_ERR_ARG, "model cuts do not match its position");
    // the neighbours along each axis share the other axis' size
    for (int o = 0; o < (int)g->mem.size(); ++o) {
        const mom6b_model* q = g->mem[o].m;
        if (!q) continue;
        const int ox = o / g->py, oy = o % g->py;
        if ((ox == x && q->D.n1 != m->D.n1) || (oy == y && q->D.n2 != m->D.n2))
            return fail(MOM6B_ERR_ARG, "subdomain sizes do not tile the layout");
    }
    g->mem[rank].m = m;
    g->ctx.push_back(std::make_unique<mom6b_halo_group::Ctx>(mom6b_halo_group::Ctx{g, rank}));
    return mom6b_set_exchange(m, group_exchange, g->ctx.back().get());
}

extern "C" void mom6b_halo_group_destroy(mom6b_halo_group* g) { delete g; }

extern "C" int mom6b_set_hor_visc(mom6b_model* m, const mom6b_hor_visc* o)
{
    if (!m || !o) return fail(MOM6B_ERR_ARG, "null argument");
    const bool plain = o->laplacian && !o->biharmonic && !o->smagorinsky && !o->leith &&
                       !o->no_slip && !o->better_bound && !o->modified_leith;
    if (!plain && m->cfg.precision != MOM6B_FP64)
        return fail(MOM6B_ERR_STATE, "the hor_visc schemes are built for the FP64 form");
    CK(cudaSetDevice(m->cfg.device));
    CK(cudaStreamSynchronize(m->s3d));
    HorViscGen& P = m->hvp;
    P.lap = o->laplacian != 0;
    P.bih = o->biharmonic != 0;
    P.smag_kh = o->smagorinsky && P.lap;
    P.smag_ah = o->smagorinsky && P.bih;
    P.leith_kh = o->leith != 0;
    P.leith_ah = o->leith && P.bih;
    P.no_slip = o->no_slip != 0;
    P.bb = o->better_bound != 0;
    P.mod_leith = o->modified_leith != 0;
    P.Kh_bg = m->cfg.Kh;
    P.Ah_bg = o->Ah;
    P.Kh_bg_min = 0.0;
    P.h_neglect = step_hv_neglect();
    if (!plain && !m->hv_du) {
        cudaError_t e = cudaSuccess;
        const HostGrid& g = *m->grid;
        const size_t n2 = (size_t)m->D.plane, n3 = n2 * m->D.nk;
        m->hv_du = dalloc(m, n3, &e);
        m->hv_dv = dalloc(m, n3, &e);
        // hor_visc_init (mom6_hor_visc_serial.F90:207-268)
        std::vector<double> a[10];
        for (auto& x : a) x.resize(n2);
        const double Smag_Lap_const = 0.15, Smag_bi_const = 0.06, Leith_const = 1.0;
        for (size_t p = 0; p < n2; ++p) {
            const double h2 = g.areaT[p], h3 = std::sqrt(h2) * h2, h4 = h2 * h2;
            a[0][p] = 0.25 * h2 / 1.0;
            a[1][p] = 0.0625 * h4 / 1.0;
            a[2][p] = Smag_Lap_const * Smag_Lap_const * h2;
            a[3][p] = Smag_bi_const * Smag_bi_const * h4;
            a[4][p] = Leith_const * h3;
            a[5][p] = Leith_const * h3 * h3;
            a[6][p] = g.IdxCu[p] * g.IdxCu[p] * g.IdyCu[p];
            a[7][p] = g.IdxCu[p] * g.IdyCu[p] * g.IdyCu[p];
            a[8][p] = g.IdxCv[p] * g.IdxCv[p] * g.IdyCv[p];
            a[9][p] = g.IdxCv[p] * g.IdyCv[p] * g.IdyCv[p];
        }
        const double** dst[10] = {&P.Kh_Max, &P.Ah_Max, &P.L2c, &P.Bc, &P.L3c, &P.B6c,
                                  &P.Idx2dyCu, &P.Idxdy2u, &P.Idx2dyCv, &P.Idxdy2v};
        double* sdst[10] = {&P.sKh_Max, &P.sAh_Max, &P.sL2c, &P.sBc, &P.sL3c, &P.sB6c,
                            &P.sIdx2dyCu, &P.sIdxdy2u, &P.sIdx2dyCv, &P.sIdxdy2v};
        // uniform over the points the kernel reads ([1, n1-1] x [1, n2-1])
        P.uni = 1;
        for (int q = 0; q < 10; ++q) {
            *sdst[q] = a[q][g.at(1, 1)];
            for (int j = 1; j <= g.n2 - 1 && P.uni; ++j)
                for (int i = 1; i <= g.n1 - 1; ++i)
                    if (a[q][g.at(i, j)] != *sdst[q]) { P.uni = 0; break; }
        }
        for (int q = 0; q < 10; ++q) {
            double* d = dalloc(m, n2, &e);
            if (e != cudaSuccess) break;
            e = cudaMemcpy(d, a[q].data(), n2 * sizeof(double), cudaMemcpyHostToDevice);
            *dst[q] = d;
        }
        if (e != cudaSuccess) return fail(MOM6B_ERR_NOMEM, "hor_visc scheme buffers");
    }
    m->hvgen = !plain;
    invalidate_graph(m);
    return MOM6B_OK;
}

extern "C" int mom6b_set_visc_remnant(mom6b_model* m, int on)
{
    if (!m) return fail(MOM6B_ERR_ARG, "null model");
    if (on && m->cfg.precision != MOM6B_FP64)
        return fail(MOM6B_ERR_STATE, "the viscous remnant is built for the FP64 form");
    CK(cudaSetDevice(m->cfg.device));
    CK(cudaStreamSynchronize(m->s3d));
    if (on && !m->visc_rem_u) {
        cudaError_t e = cudaSuccess;
        const size_t n3 = (size_t)m->D.plane * m->D.nk;
        m->visc_rem_u = dalloc(m, n3, &e);
        m->visc_rem_v = dalloc(m, n3, &e);
        if (e != cudaSuccess) return fail(MOM6B_ERR_NOMEM, "viscous remnant buffers");
        // points outside every vertvisc column keep visc_rem = 1
        std::vector<double> one(n3, 1.0);
        CK(cudaMemcpy(m->visc_rem_u, one.data(), n3 * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(m->visc_rem_v, one.data(), n3 * sizeof(double), cudaMemcpyHostToDevice));
    }
    m->remnant = on != 0;
    invalidate_graph(m);
    return MOM6B_OK;
}

extern "C" int mom6b_continuity_pass(mom6b_model* m, int dir, double dt)
{
    if (!m || (dir != 0 && dir != 1)) return fail(MOM6B_ERR_ARG, "bad argument");
    if (m->cfg.precision != MOM6B_FP64) return fail(MOM6B_ERR_STATE, "FP64 form only");
    if (dir == 1 && !m->hZ) return fail(MOM6B_ERR_STATE, "enable the meridional pass first");
    CK(cudaSetDevice(m->cfg.device));
    cudaStream_t s = m->s3d;
    const double h_min = step_h_min();
    if (dir == 0) {
        ContOut O{m->hA, m->uh, m->h_u, m->FA_u_W0, m->FA_u_WW, m->FA_u_E0,
                  m->FA_u_EE, m->uBT_WW, m->uBT_EE, m->du_cor};
        CK(timed(m, s, "continuity", [&] {
            return launch_continuity(m->D, m->M, m->u, m->h0, m->hW, m->hE, m->uhbt0, O,
                                     m->uh_ovl, dt, h_min, s,
                                     m->remnant ? m->visc_rem_u : nullptr); }));
    } else {
        ContOut O{m->hA, m->vh, m->h_v, m->FA_v_S0, m->FA_v_SS, m->FA_v_N0, m->FA_v_NN,
                  m->vBT_SS, m->vBT_NN, m->dv_cor};
        CK(timed(m, s, "continuity", [&] {
            return launch_continuity_y(m->D, m->M, m->v, m->h0, m->hW, m->hE, m->uhbt0, O,
                                       m->vh_ovl, dt, h_min, s,
                                       m->remnant ? m->visc_rem_v : nullptr); }));
    }
    CK(cudaStreamSynchronize(s));
    return MOM6B_OK;
}

// the computational domain of field f <-> a column-major host block
static int comp_domain(mom6b_model* m, int f, std::vector<double>& full, int* ni, int* nj,
                       int* nk)
{
    bool is3d, w;
    if (!field_ptr(m, f, &is3d, &w)) return fail(MOM6B_ERR_ARG, "unknown field id");
    const HostGrid& g = *m->grid;
    *ni = g.ie - g.is + 1;
    *nj = g.je - g.js + 1;
    *nk = is3d ? g.nk : 0;
    full.resize(mom6b_field_size(m, f));
    return MOM6B_OK;
}

extern "C" int mom6b_write_field_bin(mom6b_model* m, int f, const char* path)
{
    if (!m || !path) return fail(MOM6B_ERR_ARG, "null argument");
    std::vector<double> full;
    int ni, nj, nk;
    if (int rc = comp_domain(m, f, full, &ni, &nj, &nk)) return rc;
    if (int rc = mom6b_get_field(m, f, full.data(), full.size())) return rc;
    const HostGrid& g = *m->grid;
    const int nl = nk > 0 ? nk : 1;
    std::vector<double> comp((size_t)ni * nj * nl);
    for (int k = 0; k < nl; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i)
                comp[((size_t)k * nj + j) * ni + i] =
                    full[(size_t)k * g.plane + (size_t)(g.js - 1 + j) * g.n1 + (g.is - 1 + i)];
    if (diag_write_bin(path, comp.data(), ni, nj, nk) != 0)
        return fail(MOM6B_ERR_ARG, std::string("cannot write ") + path);
    return MOM6B_OK;
}

extern "C" int mom6b_read_field_bin(mom6b_model* m, int f, const char* path)
{
    if (!m || !path) return fail(MOM6B_ERR_ARG, "null argument");
    std::vector<double> full;
    int ni, nj, nk;
    if (int rc = comp_domain(m, f, full, &ni, &nj, &nk)) return rc;
    const int nl = nk > 0 ? nk : 1;
    std::vector<double> comp((size_t)ni * nj * nl);
    const int r = diag_read_bin(path, comp.data(), ni, nj, nk);
    if (r == -2) return fail(MOM6B_ERR_ARG, std::string("dimensions in ") + path + " do not match");
    if (r != 0) return fail(MOM6B_ERR_ARG, std::string("cannot read ") + path);
    if (int rc = mom6b_get_field(m, f, full.data(), full.size())) return rc;
    const HostGrid& g = *m->grid;
    for (int k = 0; k < nl; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i)
                full[(size_t)k * g.plane + (size_t)(g.js - 1 + j) * g.n1 + (g.is - 1 + i)] =
                    comp[((size_t)k * nj + j) * ni + i];
    return mom6b_set_field(m, f, full.data(), full.size());
}

struct mom6b_ensemble {
    std::vector<mom6b_model*> doms;
    std::vector<EnsDomain> host;
    EnsDomain* d_doms = nullptr;
    EnsTuning T{0, 5, 128, 4, 128, 128, 64};
    bool uni = true, uni_bt = true;
    int kmax = 0, max_nstep = 0, device = 0;
    // block tables of the current tuning (device) and their totals
    int *st_tend = nullptr, *st_vv = nullptr, *st_ppm = nullptr, *st_faces = nullptr;
    int *st_halo[4] = {nullptr, nullptr, nullptr, nullptr};
    int tot_tend = 0, tot_vv = 0, tot_ppm = 0, tot_faces = 0, tot_halo[4] = {0, 0, 0, 0};
    EnsBtGeo* d_geo = nullptr;
    int* d_tstart = nullptr;
    int ntiles = 0, max_tw = 0, max_th = 0;
    BTWork ctl{};
    int max_tiles_alloc = 0;
    std::vector<void*> allocs;
    std::vector<void*> plan_allocs;
    cudaStream_t s = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int use_graph = 1;
    int64_t launches = 0, launches_per_step = 0;
};

static void ens_free_plan(mom6b_ensemble* e)
{
    for (void* p : e->plan_allocs) cudaFree(p);
    e->plan_allocs.clear();
    if (e->exec) { cudaGraphExecDestroy(e->exec); e->exec = nullptr; }
    if (e->graph) { cudaGraphDestroy(e->graph); e->graph = nullptr; }
}

static void ens_free(mom6b_ensemble* e)
{
    if (e->s) cudaStreamSynchronize(e->s);
    ens_free_plan(e);
    for (void* p : e->allocs) cudaFree(p);
    e->allocs.clear();
    for (mom6b_model* m : e->doms) mom6b_destroy(m);
    e->doms.clear();
    if (e->s) cudaStreamDestroy(e->s);
    e->s = nullptr;
}

// Upload a block table built from per-job block counts; returns the total.
static int ens_table(mom6b_ensemble* e, const std::vector<long long>& counts, int** dst,
                     int* total)
{
    std::vector<int> st(counts.size() + 1, 0);
    long long acc = 0;
    for (size_t q = 0; q < counts.size(); ++q) {
        st[q] = (int)acc;
        acc += counts[q];
        if (acc > 2147483647LL) return fail(MOM6B_ERR_ARG, "ensemble grid too large");
    }
    st[counts.size()] = (int)acc;
    void* p = nullptr;
    CK(cudaMalloc(&p, st.size() * sizeof(int)));
    e->plan_allocs.push_back(p);
    CK(cudaMemcpy(p, st.data(), st.size() * sizeof(int), cudaMemcpyHostToDevice));
    *dst = (int*)p;
    *total = (int)acc;
    return MOM6B_OK;
}

// Block tables and barotropic tiles for the current tuning.
static int ens_plan(mom6b_ensemble* e)
{
    ens_free_plan(e);
    const int n = (int)e->doms.size();
    const EnsTuning& T = e->T;
    std::vector<long long> ct(n), cv(n), cp(n), cf(n);
    for (int d = 0; d < n; ++d) {
        const Dims& D = e->host[d].D;
        ct[d] = ens_blocks_tendency(D, T);
        cv[d] = ens_blocks_vertvisc(D, T);
        cp[d] = ens_blocks_ppm(D, T);
        cf[d] = ens_blocks_faces(D, T);
    }
    if (int rc = ens_table(e, ct, &e->st_tend, &e->tot_tend)) return rc;
    if (int rc = ens_table(e, cv, &e->st_vv, &e->tot_vv)) return rc;
    if (int rc = ens_table(e, cp, &e->st_ppm, &e->tot_ppm)) return rc;
    if (int rc = ens_table(e, cf, &e->st_faces, &e->tot_faces)) return rc;
    for (int w = 0; w < 4; ++w) {
        const int F = w == 3 ? 1 : 3;
        std::vector<long long> ch((size_t)n * F);
        for (int d = 0; d < n; ++d)
            for (int f = 0; f < F; ++f)
                ch[(size_t)d * F + f] = e->host[d].bc_fill ? ens_blocks_halo(e->host[d].D, w) : 0;
        if (int rc = ens_table(e, ch, &e->st_halo[w], &e->tot_halo[w])) return rc;
    }
    std::vector<EnsBtGeo> geo(n);
    std::vector<int> tst(n + 1);
    int nt = 0, mtw = 0, mth = 0;
    for (int d = 0; d < n; ++d) {
        geo[d] = ens_bt_geometry(e->host[d].D, T.bt_tile);
        geo[d].t0 = nt;
        tst[d] = nt;
        nt += geo[d].nbx * geo[d].nby;
        mtw = std::max(mtw, geo[d].tw);
        mth = std::max(mth, geo[d].th);
    }
    tst[n] = nt;
    if (nt > e->max_tiles_alloc) return fail(MOM6B_ERR_ARG, "too many barotropic tiles");
    void* pg = nullptr;
    void* pt = nullptr;
    CK(cudaMalloc(&pg, n * sizeof(EnsBtGeo)));
    e->plan_allocs.push_back(pg);
    CK(cudaMalloc(&pt, (n + 1) * sizeof(int)));
    e->plan_allocs.push_back(pt);
    CK(cudaMemcpy(pg, geo.data(), n * sizeof(EnsBtGeo), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(pt, tst.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice));
    e->d_geo = (EnsBtGeo*)pg;
    e->d_tstart = (int*)pt;
    e->ntiles = nt;
    e->max_tw = mtw;
    e->max_th = mth;
    return MOM6B_OK;
}

// One launch of phase `ph` (0..13 in step order); counts the launch.
static int ens_launch(mom6b_ensemble* e, int ph)
{
    const int n = (int)e->doms.size();
    cudaStream_t s = e->s;
    cudaError_t r = cudaSuccess;
    switch (ph) {
    case 0: case 5:
        r = launch_ens_tendency(e->d_doms, e->st_tend, n, e->tot_tend, ph == 5, e->T, e->uni, s);
        break;
    case 1: case 6:
        r = launch_ens_vertvisc(e->d_doms, e->st_vv, n, e->tot_vv, ph == 6, e->kmax, e->T, s);
        break;
    case 2: case 7:
        r = launch_ens_ppm(e->d_doms, e->st_ppm, n, e->tot_ppm, ph == 7, e->T, s);
        break;
    case 3: case 8:
        r = launch_ens_faces(e->d_doms, e->st_faces, n, e->tot_faces, ph == 8, e->T, s);
        break;
    case 4: case 9:
        r = launch_ens_halo(e->d_doms, e->st_halo[ph == 9], 3 * n, e->tot_halo[ph == 9],
                            ph == 9, s);
        break;
    case 10: case 12:
        r = launch_ens_btstep(e->d_doms, e->d_geo, e->d_tstart, n, e->ntiles, e->max_tw,
                              e->max_th, ph == 12, e->max_nstep, e->ctl, e->uni_bt, s);
        break;
    case 11:
        r = launch_ens_halo(e->d_doms, e->st_halo[2], 3 * n, e->tot_halo[2], 2, s);
        break;
    case 13:
        r = launch_ens_halo(e->d_doms, e->st_halo[3], n, e->tot_halo[3], 3, s);
        break;
    default: return fail(MOM6B_ERR_ARG, "unknown ensemble phase");
    }
    if (r != cudaSuccess) return fail(MOM6B_ERR_CUDA, std::string("ensemble launch: ") + cudaGetErrorString(r));
    ++e->launches;
    return MOM6B_OK;
}

static bool ens_phase_active(const mom6b_ensemble* e, int ph)
{
    if (ph == 4 || ph == 9) return e->tot_halo[ph == 9] > 0;
    if (ph == 11) return e->tot_halo[2] > 0;
    if (ph == 13) return e->tot_halo[3] > 0;
    return true;
}

static int ens_enqueue(mom6b_ensemble* e)
{
    for (int ph = 0; ph < 14; ++ph)
        if (ens_phase_active(e, ph))
            if (int rc = ens_launch(e, ph)) return rc;
    return MOM6B_OK;
}

extern "C" int mom6b_ensemble_create(int n, const mom6b_config* cfgs, mom6b_ensemble** out)
{
    if (!out || !cfgs || n < 1) return fail(MOM6B_ERR_ARG, "bad argument");
    *out = nullptr;
    auto e = std::make_unique<mom6b_ensemble>();
    e->device = cfgs[0].device;
    for (int d = 0; d < n; ++d) {
        if (cfgs[d].precision != MOM6B_MIXED)
            return fail(MOM6B_ERR_ARG, "ensemble domains run the mixed form (precision MOM6B_MIXED)");
        if (cfgs[d].device != e->device)
            return fail(MOM6B_ERR_ARG, "ensemble domains share one device");
        if (cfgs[d].nk > 256) return fail(MOM6B_ERR_ARG, "ensemble domains need nk <= 256");
    }
    CK(cudaSetDevice(e->device));
    for (int d = 0; d < n; ++d) {
        mom6b_config c = cfgs[d];
        c.use_graph = 0;
        mom6b_model* m = nullptr;
        int rc = mom6b_create(&c, &m);
        if (rc) { ens_free(e.get()); return rc; }
        e->doms.push_back(m);
    }
    // descriptors
    size_t max_tiles = 0;
    for (int d = 0; d < n; ++d) {
        mom6b_model* m = e->doms[d];
        const mom6b_config& c = m->cfg;
        EnsDomain E{};
        E.D = m->D; E.M = m->M; E.U = m->U;
        auto F = [](double* p) { return (float*)p; };
        E.u = F(m->u); E.v = F(m->v); E.hA = F(m->hA); E.hB = F(m->hB); E.h0 = F(m->h0);
        E.up = F(m->up); E.vp = F(m->vp); E.uh = F(m->uh); E.hW = F(m->hW); E.hE = F(m->hE);
        E.h_u = F(m->h_u);
        void* po = nullptr;
        if (cudaMalloc(&po, ens_ovl_floats(m->D) * sizeof(float) + 16) != cudaSuccess) {
            ens_free(e.get());
            return fail(MOM6B_ERR_NOMEM, "device allocation failed");
        }
        e->allocs.push_back(po);
        E.ovl = (float*)po;
        E.uhbt0 = m->uhbt0; E.taux_bot = m->taux_bot; E.tauy_bot = m->tauy_bot;
        E.O2 = ContOut{nullptr, nullptr, nullptr, m->FA_u_W0, m->FA_u_WW, m->FA_u_E0,
                       m->FA_u_EE, m->uBT_WW, m->uBT_EE, m->du_cor};
        E.eta = m->eta; E.ubt = m->ubt; E.vbt = m->vbt;
        E.ubt_av = m->ubt_av; E.vbt_av = m->vbt_av; E.eta_av = m->eta_av;
        E.W = m->bt;
        E.VV = step_vv_params(c);
        E.P = step_bt_params(c);
        E.dt = c.dt;
        E.h_min = step_h_min();
        E.hv_neglect = (float)step_hv_neglect();
        E.bc_fill = c.bc_fill;
        e->host.push_back(E);
        e->uni = e->uni && m->U.valid;
        e->uni_bt = e->uni_bt && m->U.valid_bt;
        e->kmax = std::max(e->kmax, m->D.nk);
        e->max_nstep = std::max(e->max_nstep, c.bt_nsteps);
        EnsBtGeo g = ens_bt_geometry(m->D, 32);
        max_tiles += (size_t)g.nbx * g.nby;
    }
    {
        void* p = nullptr;
        CK(cudaMalloc(&p, n * sizeof(EnsDomain)));
        e->allocs.push_back(p);
        CK(cudaMemcpy(p, e->host.data(), n * sizeof(EnsDomain), cudaMemcpyHostToDevice));
        e->d_doms = (EnsDomain*)p;
        // barrier words, status and one flag per tile (the smallest tile edge)
        void* pc = nullptr;
        const size_t bytes = 64 + max_tiles * sizeof(unsigned int);
        CK(cudaMalloc(&pc, bytes));
        e->allocs.push_back(pc);
        CK(cudaMemset(pc, 0, bytes));
        e->ctl.bar_count = (unsigned int*)pc;
        e->ctl.bar_gen = (unsigned int*)pc + 4;
        e->ctl.status = (int*)pc + 8;
        e->ctl.tile_flag = (unsigned int*)pc + 16;
        e->max_tiles_alloc = (int)max_tiles;
    }
    CK(cudaStreamCreateWithFlags(&e->s, cudaStreamNonBlocking));
    if (int rc = ens_plan(e.get())) { ens_free(e.get()); return rc; }
    *out = e.release();
    return MOM6B_OK;
}

extern "C" int mom6b_ensemble_destroy(mom6b_ensemble* e)
{
    if (!e) return MOM6B_OK;
    cudaSetDevice(e->device);
    ens_free(e);
    delete e;
    return MOM6B_OK;
}

extern "C" int mom6b_ensemble_size(const mom6b_ensemble* e)
{
    return e ? (int)e->doms.size() : 0;
}

extern "C" int mom6b_ensemble_step(mom6b_ensemble* e, int nsteps)
{
    if (!e || nsteps < 0) return fail(MOM6B_ERR_ARG, "bad argument");
    CK(cudaSetDevice(e->device));
    if (e->use_graph) {
        if (!e->exec) {
            int64_t before = e->launches;
            CK(cudaStreamBeginCapture(e->s, cudaStreamCaptureModeThreadLocal));
            int rc = ens_enqueue(e);
            cudaGraph_t g = nullptr;
            cudaError_t r = cudaStreamEndCapture(e->s, &g);
            if (rc) { if (g) cudaGraphDestroy(g); return rc; }
            if (r != cudaSuccess) return fail(MOM6B_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(r));
            e->graph = g;
            CK(cudaGraphInstantiate(&e->exec, g, 0));
            e->launches_per_step = e->launches - before;
            e->launches = before;
        }
        for (int k = 0; k < nsteps; ++k) {
            CK(cudaGraphLaunch(e->exec, e->s));
            e->launches += e->launches_per_step;
        }
        return MOM6B_OK;
    }
    for (int k = 0; k < nsteps; ++k)
        if (int rc = ens_enqueue(e)) return rc;
    return MOM6B_OK;
}

static int ens_check_status(mom6b_ensemble* e)
{
    int st = 0;
    CK(cudaMemcpy(&st, e->ctl.status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st != kDevOk) {
        cudaMemset(e->ctl.status, 0, sizeof(int));
        cudaMemset(e->ctl.bar_count, 0, sizeof(unsigned int));
        return fail(MOM6B_ERR_TIMEOUT, "ensemble barotropic wait timed out");
    }
    return MOM6B_OK;
}

extern "C" int mom6b_ensemble_synchronize(mom6b_ensemble* e)
{
    if (!e) return fail(MOM6B_ERR_ARG, "null ensemble");
    CK(cudaSetDevice(e->device));
    CK(cudaStreamSynchronize(e->s));
    return ens_check_status(e);
}

extern "C" int mom6b_ensemble_stream(mom6b_ensemble* e, void** stream)
{
    if (!e || !stream) return fail(MOM6B_ERR_ARG, "null argument");
    *stream = (void*)e->s;
    return MOM6B_OK;
}

extern "C" int64_t mom6b_ensemble_launch_count(const mom6b_ensemble* e)
{
    return e ? e->launches : 0;
}

extern "C" mom6b_model* mom6b_ensemble_member(mom6b_ensemble* e, int d)
{
    if (!e || d < 0 || d >= (int)e->doms.size()) return nullptr;
    return e->doms[d];
}

extern "C" int mom6b_ensemble_get_field(mom6b_ensemble* e, int d, int field, double* host,
                                        size_t count)
{
    if (!e || d < 0 || d >= (int)e->doms.size()) return fail(MOM6B_ERR_ARG, "bad domain index");
    if (int rc = mom6b_ensemble_synchronize(e)) return rc;
    return mom6b_get_field(e->doms[d], field, host, count);
}

// Tuning as 7 ints: tendency tile index, tendency layers per CTA, vertvisc
// threads per CTA, vertvisc prefetch depth, PPM threads per CTA, faces per
// CTA + 1, barotropic tile edge.
static bool ens_tuning_valid(const EnsTuning& T)
{
    auto in = [](int v, std::initializer_list<int> set) {
        for (int x : set) if (v == x) return true;
        return false;
    };
    return T.tend >= 0 && T.tend < 4 && T.tend_kc >= 1 && T.tend_kc <= 16 &&
           in(T.vv_nb, {64, 128, 256}) && in(T.vv_ch, {2, 4}) && in(T.ppm_nb, {128, 256}) &&
           in(T.faces_nb, {64, 128, 256}) && in(T.bt_tile, {32, 48, 64});
}

extern "C" int mom6b_ensemble_get_tuning(const mom6b_ensemble* e, int* out7)
{
    if (!e || !out7) return fail(MOM6B_ERR_ARG, "null argument");
    const EnsTuning& T = e->T;
    int v[7] = {T.tend, T.tend_kc, T.vv_nb, T.vv_ch, T.ppm_nb, T.faces_nb, T.bt_tile};
    std::memcpy(out7, v, sizeof(v));
    return MOM6B_OK;
}

extern "C" int mom6b_ensemble_set_tuning(mom6b_ensemble* e, const int* in7)
{
    if (!e || !in7) return fail(MOM6B_ERR_ARG, "null argument");
    EnsTuning T{in7[0], in7[1], in7[2], in7[3], in7[4], in7[5], in7[6]};
    if (!ens_tuning_valid(T)) return fail(MOM6B_ERR_ARG, "tuning value outside the supported set");
    CK(cudaSetDevice(e->device));
    CK(cudaStreamSynchronize(e->s));
    e->T = T;
    return ens_plan(e);
}

// Device copies of every array a step rewrites, to undo the tuning trials.
struct EnsSnapshot {
    std::vector<std::pair<void*, void*>> saved;  // (live, copy)
    std::vector<size_t> bytes;
};

static int ens_snapshot(mom6b_ensemble* e, EnsSnapshot& S)
{
    for (mom6b_model* m : e->doms) {
        const size_t n3 = m->grid->plane * (size_t)m->grid->nk, n2 = m->grid->plane;
        const size_t b3 = n3 * sizeof(float), b2 = n2 * sizeof(double);
        void* live[] = {m->u, m->v, m->hA, m->hB, m->up, m->vp, m->uh, m->h_u, m->hW, m->hE,
                        m->eta, m->ubt, m->vbt, m->ubt_av, m->vbt_av, m->eta_av,
                        m->taux_bot, m->tauy_bot, m->FA_u_W0, m->FA_u_WW, m->FA_u_E0,
                        m->FA_u_EE, m->uBT_WW, m->uBT_EE, m->du_cor};
        for (int q = 0; q < 25; ++q) {
            const size_t b = q < 10 ? b3 : b2;
            void* c = nullptr;
            CK(cudaMalloc(&c, b));
            S.saved.push_back({live[q], c});
            S.bytes.push_back(b);
            CK(cudaMemcpyAsync(c, live[q], b, cudaMemcpyDeviceToDevice, e->s));
        }
    }
    CK(cudaStreamSynchronize(e->s));
    return MOM6B_OK;
}

static int ens_restore(mom6b_ensemble* e, EnsSnapshot& S)
{
    for (size_t q = 0; q < S.saved.size(); ++q)
        CK(cudaMemcpyAsync(S.saved[q].first, S.saved[q].second, S.bytes[q],
                           cudaMemcpyDeviceToDevice, e->s));
    CK(cudaStreamSynchronize(e->s));
    for (auto& p : S.saved) cudaFree(p.second);
    S.saved.clear();
    return MOM6B_OK;
}

// Time `reps` launches of phase ph under the current plan; the best average
// of three rounds, in ms.
static int ens_time_phase(mom6b_ensemble* e, int ph, int reps, double* ms)
{
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    double best = 1e30;
    if (int rc = ens_launch(e, ph)) return rc;   // warm-up
    for (int round = 0; round < 3; ++round) {
        CK(cudaEventRecord(a, e->s));
        for (int r = 0; r < reps; ++r)
            if (int rc = ens_launch(e, ph)) return rc;
        CK(cudaEventRecord(b, e->s));
        CK(cudaEventSynchronize(b));
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, a, b));
        best = std::min(best, (double)t / reps);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (int rc = ens_check_status(e)) return rc;
    *ms = best;
    return MOM6B_OK;
}

// The autotuner: for each phase group, time every candidate launch shape on
// the ensemble's own domains (state saved before and restored after) and keep
// the fastest.  out_ms (optional, 5 entries) receives the best time of the
// tendency, vertvisc, PPM, faces and barotropic launches.
extern "C" int mom6b_ensemble_autotune(mom6b_ensemble* e, int reps, double* out_ms)
{
    if (!e) return fail(MOM6B_ERR_ARG, "null ensemble");
    if (reps < 1) reps = 1;
    CK(cudaSetDevice(e->device));
    CK(cudaStreamSynchronize(e->s));
    EnsSnapshot S;
    if (int rc = ens_snapshot(e, S)) return rc;
    EnsTuning best = e->T;
    double tbest[5] = {0, 0, 0, 0, 0};
    auto sweep = [&](int slot, int ph, const std::vector<EnsTuning>& cands) -> int {
        double bt = 1e30;
        EnsTuning bc = best;
        for (const EnsTuning& c : cands) {
            e->T = c;
            if (int rc = ens_plan(e)) return rc;
            double ms = 0.0;
            if (int rc = ens_time_phase(e, ph, reps, &ms)) return rc;
            if (ms < bt) { bt = ms; bc = c; }
        }
        best = bc;
        tbest[slot] = bt;
        return MOM6B_OK;
    };
    std::vector<EnsTuning> c;
    for (int t = 0; t < 4; ++t)
        for (int kc : {3, 5, 8}) { EnsTuning x = best; x.tend = t; x.tend_kc = kc; c.push_back(x); }
    int rc = sweep(0, 0, c);
    if (!rc) {
        c.clear();
        for (int nb : {64, 128, 256})
            for (int ch : {2, 4}) { EnsTuning x = best; x.vv_nb = nb; x.vv_ch = ch; c.push_back(x); }
        rc = sweep(1, 1, c);
    }
    if (!rc) {
        c.clear();
        for (int nb : {128, 256}) { EnsTuning x = best; x.ppm_nb = nb; c.push_back(x); }
        rc = sweep(2, 2, c);
    }
    if (!rc) {
        c.clear();
        for (int nb : {64, 128, 256}) { EnsTuning x = best; x.faces_nb = nb; c.push_back(x); }
        rc = sweep(3, 3, c);
    }
    if (!rc) {
        c.clear();
        for (int t : {32, 48, 64}) { EnsTuning x = best; x.bt_tile = t; c.push_back(x); }
        rc = sweep(4, 10, c);
    }
    int rr = ens_restore(e, S);
    e->T = best;
    int rp = ens_plan(e);
    if (rc) return rc;
    if (rr) return rr;
    if (rp) return rp;
    if (out_ms) std::memcpy(out_ms, tbest, sizeof(tbest));
    return MOM6B_OK;
}

// ===========================================================================
// Learned barotropic surrogate: training, control and the network's own ABI
// ===========================================================================
static uint64_t sur_hash(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Barotropic initial state k of the training set: a Gaussian eta bump whose
// amplitude (0.05 .. 0.15 m), centre (the middle half of the basin in each
// direction) and radius (120 .. 280 km) are drawn from (seed, k); ubt = vbt = 0
// as in the configured beta-plane state.
static void sur_initial_eta(const mom6b_model* m, uint64_t seed, int k, std::vector<double>& eta)
{
    const HostGrid& g = *m->grid;
    uint64_t st = sur_hash(seed * 1000003ULL + (uint64_t)k);
    auto uni = [&]() {
        st = sur_hash(st);
        return (double)(st >> 11) * (1.0 / 9007199254740992.0);
    };
    const double amp = 0.1 * (0.5 + uni());
    const double cxf = 0.25 + 0.5 * uni(), cyf = 0.25 + 0.5 * uni();
    const double R = 200.0e3 * (0.6 + 0.8 * uni());
    const double Lx = (double)(g.ie - g.is + 1) * g.dx, Ly = (double)(g.je - g.js + 1) * g.dx;
    eta.assign(g.plane, 0.0);
    for (int j = g.jsd; j <= g.jed; ++j)
        for (int i = g.isd; i <= g.ied; ++i) {
            const double x = ((double)(i - g.is) + 0.5) * g.dx - cxf * Lx;
            const double y = ((double)(j - g.js) + 0.5) * g.dx - cyf * Ly;
            eta[g.at(i, j)] = amp * std::exp(-(x * x + y * y) / (R * R));
        }
}

// Shadow and training buffers (allocated once, before any capture).
static int sur_buffers(mom6b_model* m)
{
    if (m->sh_eta) return MOM6B_OK;
    cudaError_t err = cudaSuccess;
    const size_t n2 = m->grid->plane;
    m->sh_eta = dalloc(m, n2, &err);
    m->sh_ubt_av = dalloc(m, n2, &err);
    m->sh_vbt_av = dalloc(m, n2, &err);
    m->sh_eta_av = dalloc(m, n2, &err);
    m->sur_acc = dalloc(m, 4, &err);
    if (err != cudaSuccess || !m->sur_acc) return fail(MOM6B_ERR_NOMEM, "device allocation failed");
    return MOM6B_OK;
}

// channel sums over the compute domain for the normalisation
struct ChanStats {
    double n = 0, s = 0, s2 = 0;
    void add(double v) { n += 1; s += v; s2 += v * v; }
    // std, or |mean| (or 1) when the channel is constant
    float scale() const
    {
        if (n <= 0) return 1.0f;
        const double mu = s / n;
        const double var = std::max(0.0, s2 / n - mu * mu);
        const double sd = std::sqrt(var);
        if (sd > 1e-12 * std::max(std::fabs(mu), 1e-300)) return (float)sd;
        return std::fabs(mu) > 0 ? (float)std::fabs(mu) : 1.0f;
    }
};

static int sur_train_buffers(mom6b_model* m)
{
    if (m->tr_e) return MOM6B_OK;
    cudaError_t err = cudaSuccess;
    const size_t n2 = m->grid->plane;
    m->tr_e = dalloc(m, n2, &err);
    m->tr_u = dalloc(m, n2, &err);
    m->tr_v = dalloc(m, n2, &err);
    m->tr_ea = dalloc(m, n2, &err);
    m->tr_ua = dalloc(m, n2, &err);
    m->tr_va = dalloc(m, n2, &err);
    if (err != cudaSuccess || !m->tr_va) return fail(MOM6B_ERR_NOMEM, "device allocation failed");
    return MOM6B_OK;
}

// training / evaluation state k of the seeded family (synchronous)
static int sur_reset_state(mom6b_model* m, uint64_t seed, int k, cudaStream_t s)
{
    const size_t n2 = m->grid->plane;
    std::vector<double> eta;
    sur_initial_eta(m, seed, k, eta);
    CK(cudaMemcpyAsync(m->tr_e, eta.data(), n2 * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(m->tr_u, 0, n2 * sizeof(double), s));
    CK(cudaMemsetAsync(m->tr_v, 0, n2 * sizeof(double), s));
    if (m->cfg.bc_fill) CK(launch_halo_fill(m->D, m->tr_e, 1, 0, s));
    CK(cudaStreamSynchronize(s));
    return MOM6B_OK;
}

// one plain barotropic call that also leaves the averaged transports in
// bt.uhbt / bt.vhbt
static int sur_plain_call(mom6b_model* m, const double* e, const double* u, const double* v,
                          double* uo, double* vo, double* eo, cudaStream_t s)
{
    CK(launch_btstep_tavg(m->D, m->M, m->U, m->bt, step_bt_params(m->cfg), e, u, v, uo, vo, eo,
                          s));
    return MOM6B_OK;
}

static int sur_fill3(mom6b_model* m, double* e, double* u, double* v, cudaStream_t s)
{
    if (!m->cfg.bc_fill) return MOM6B_OK;
    CK(launch_halo_fill(m->D, e, 1, 0, s));
    CK(launch_halo_fill(m->D, u, 1, 1, s));
    CK(launch_halo_fill(m->D, v, 1, 2, s));
    return MOM6B_OK;
}

// Run nsteps RK2 barotropic chains of state k with the plain btstep; visit
// is called with the inputs of every call before it and after it (phase 0
// and 1, with the call's index).
template <class Visit>
static int sur_run_state(mom6b_model* m, uint64_t seed, int k, int nsteps, cudaStream_t s,
                         Visit&& visit)
{
    if (int rc = sur_reset_state(m, seed, k, s)) return rc;
    double *te = m->tr_e, *tu = m->tr_u, *tv = m->tr_v;
    double *tea = m->tr_ea, *tua = m->tr_ua, *tva = m->tr_va;
    for (int n = 0; n < nsteps; ++n) {
        if (int rc = visit(0, 2 * n, te, tu, tv)) return rc;
        if (int rc = sur_plain_call(m, te, tu, tv, tua, tva, tea, s)) return rc;
        if (int rc = visit(1, 2 * n, te, tu, tv)) return rc;
        if (int rc = sur_fill3(m, tea, tua, tva, s)) return rc;
        if (int rc = visit(0, 2 * n + 1, tea, tua, tva)) return rc;
        if (int rc = sur_plain_call(m, tea, tua, tva, tua, tva, te, s)) return rc;
        if (int rc = visit(1, 2 * n + 1, tea, tua, tva)) return rc;
        if (m->cfg.bc_fill) CK(launch_halo_fill(m->D, te, 1, 0, s));
    }
    return MOM6B_OK;
}

extern "C" int mom6b_surrogate_train(mom6b_model* m, int nstates, int nsteps, int batch,
                                     double lr, uint64_t seed, double* stats4)
{
    if (!m || nstates < 1 || nsteps < 1 || batch < 128 || batch % 8)
        return fail(MOM6B_ERR_ARG, "bad argument (batch: a multiple of 8, at least 128)");
    CK(cudaSetDevice(m->cfg.device));
    cudaStream_t s = m->s3d;
    CK(cudaStreamSynchronize(s));
    CK(cudaStreamSynchronize(m->s2d));
    const auto t0 = std::chrono::steady_clock::now();
    if (!m->sur || m->sur->B_cap < batch) {
        auto N = std::make_unique<Mlp>();
        CK(N->init(batch, seed, s));
        m->sur = std::move(N);
    }
    if (int rc = sur_buffers(m)) return rc;
    if (int rc = sur_train_buffers(m)) return rc;
    Mlp& N = *m->sur;
    const HostGrid& hg = *m->grid;
    const size_t n2 = hg.plane;
    const SurGrid g = sur_grid(m);

    // 1. normalisation from the first state's first steps: channel stds of the
    //    call inputs and of the targets over the compute domain
    {
        ChanStats cs[kMlpChannels], ts[2];
        std::vector<double> a(n2), b(n2), c(n2), tu_h(n2), tv_h(n2);
        auto visit = [&](int phase, int, const double* e, const double* u, const double* v) -> int {
            if (phase == 0) {
                CK(cudaStreamSynchronize(s));
                CK(cudaMemcpy(a.data(), e, n2 * sizeof(double), cudaMemcpyDeviceToHost));
                CK(cudaMemcpy(b.data(), u, n2 * sizeof(double), cudaMemcpyDeviceToHost));
                CK(cudaMemcpy(c.data(), v, n2 * sizeof(double), cudaMemcpyDeviceToHost));
                return MOM6B_OK;
            }
            CK(cudaStreamSynchronize(s));
            CK(cudaMemcpy(tu_h.data(), m->bt.uhbt, n2 * sizeof(double), cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(tv_h.data(), m->bt.vhbt, n2 * sizeof(double), cudaMemcpyDeviceToHost));
            for (int j = hg.js; j <= hg.je; ++j)
                for (int i = hg.is; i <= hg.ie; ++i) {
                    const size_t p = hg.at(i, j);
                    cs[0].add(a[p]); cs[1].add(b[p]); cs[2].add(c[p]);
                    ts[0].add(tu_h[p]); ts[1].add(tv_h[p]);
                }
            return MOM6B_OK;
        };
        if (int rc = sur_run_state(m, seed, 0, std::min(nsteps, 10), s, visit)) return rc;
        std::vector<double> cor(n2);
        CK(cudaMemcpy(cor.data(), m->M.CoriolisBu, n2 * sizeof(double), cudaMemcpyDeviceToHost));
        for (int j = hg.js; j <= hg.je; ++j)
            for (int i = hg.is; i <= hg.ie; ++i) cs[6].add(cor[hg.at(i, j)]);
        cs[5].add(g.depth);
        for (int q = 0; q < kMlpChannels; ++q) N.feat_std[q] = cs[q].scale();
        N.targ_std[0] = ts[0].scale();
        N.targ_std[1] = ts[1].scale();
        float nrm[16] = {0};
        for (int q = 0; q < kMlpChannels; ++q) nrm[q] = 1.0f / N.feat_std[q];
        nrm[7] = N.targ_std[0];
        nrm[8] = N.targ_std[1];
        CK(cudaMemcpy(N.d_norm, nrm, sizeof(nrm), cudaMemcpyHostToDevice));
    }

    // 2. training: every barotropic call of every step of every state gives one
    //    batch of sampled columns and one Adam step
    const int64_t total = (int64_t)nstates * nsteps * 2;
    float* dloss = nullptr;
    CK(cudaMalloc(&dloss, (size_t)total * sizeof(float)));
    std::unique_ptr<float, decltype(&cudaFree)> dloss_guard(dloss, cudaFree);
    int64_t q = 0;
    uint64_t cseed = 0;
    auto train_visit = [&](int phase, int, const double* e, const double* u,
                           const double* v) -> int {
        if (phase == 0) {   // features of the inputs, before the call overwrites them
            cseed = sur_hash(seed ^ (0x5DEECE66DULL * (uint64_t)(q + 1)));
            CK(launch_sur_features_train(g, BtInputs{e, u, v}, N.d_norm, N.gacc, batch, cseed, N.X,
                                         N.XT, N.amp, s));
            return MOM6B_OK;
        }
        CK(launch_sur_targets(g, m->bt.uhbt, m->bt.vhbt, N.d_norm, N.amp, batch, cseed, N.Y, s));
        CK(N.train_step(batch, (float)lr, s));
        CK(cudaMemcpyAsync(dloss + q, N.loss, sizeof(float), cudaMemcpyDeviceToDevice, s));
        ++q;
        return MOM6B_OK;
    };
    for (int k = 0; k < nstates; ++k)
        if (int rc = sur_run_state(m, seed, k, nsteps, s, train_visit)) return rc;
    CK(cudaStreamSynchronize(s));
    int gerr = 0;
    CK(cudaMemcpy(&gerr, N.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (gerr) return fail(MOM6B_ERR_TIMEOUT, "tensor-core pipeline wait timed out");
    if (int rc = check_status(m)) return rc;
    std::vector<float> L((size_t)total);
    CK(cudaMemcpy(L.data(), dloss, (size_t)total * sizeof(float), cudaMemcpyDeviceToHost));
    auto mean = [&](int64_t lo, int64_t hi) {
        double acc = 0.0;
        for (int64_t t = lo; t < hi; ++t) acc += L[(size_t)t];
        return hi > lo ? acc / (double)(hi - lo) : 0.0;
    };
    const int64_t w = std::min<int64_t>(total, 100);
    m->sur_loss_first = mean(0, std::min<int64_t>(total, 10));
    m->sur_loss_last = mean(total - w, total);
    m->sur_train_steps += total;
    m->sur_train_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (stats4) {
        stats4[0] = m->sur_loss_first;
        stats4[1] = m->sur_loss_last;
        stats4[2] = (double)total;
        stats4[3] = m->sur_train_s;
    }
    invalidate_graph(m);
    return MOM6B_OK;
}

// Transport error of the network on state k of the seeded family (use a k the
// training did not see): over nsteps RK2 barotropic chains of the plain
// btstep, the network predicts the averaged transports of every compute cell
// from each call's inputs.  out3: relative L2 error of the predictions over
// all calls, the same for predicting zero transport (1 when the transports
// are not all zero), calls.
extern "C" int mom6b_surrogate_eval(mom6b_model* m, uint64_t seed, int k, int nsteps,
                                    double* out3)
{
    if (!m || !out3 || nsteps < 1) return fail(MOM6B_ERR_ARG, "bad argument");
    if (!m->sur) return fail(MOM6B_ERR_STATE, "no surrogate network");
    CK(cudaSetDevice(m->cfg.device));
    cudaStream_t s = m->s3d;
    CK(cudaStreamSynchronize(s));
    if (int rc = sur_buffers(m)) return rc;
    if (int rc = sur_train_buffers(m)) return rc;
    Mlp& N = *m->sur;
    const SurGrid g = sur_grid(m);
    const int nc = (m->D.ie - m->D.is + 1) * (m->D.je - m->D.js + 1);
    CK(N.prepare_inference(nc));
    CK(cudaMemsetAsync(m->sur_acc, 0, 2 * sizeof(double), s));
    int calls = 0;
    auto visit = [&](int phase, int, const double* e, const double* u, const double* v) -> int {
        if (phase == 0) {
            CK(launch_sur_features_all(g, BtInputs{e, u, v}, N.d_norm, N.gacc, N.Xi, N.ampi, s));
            CK(N.predict(nc, s));
            return MOM6B_OK;
        }
        CK(launch_sur_transport_err(g, N.outi, N.d_norm, N.ampi, m->bt.uhbt, m->bt.vhbt,
                                    m->sur_acc, s));
        ++calls;
        return MOM6B_OK;
    };
    if (int rc = sur_run_state(m, seed, k, nsteps, s, visit)) return rc;
    double acc[2] = {0.0, 0.0};
    CK(cudaMemcpyAsync(acc, m->sur_acc, sizeof(acc), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    int gerr = 0;
    CK(cudaMemcpy(&gerr, N.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (gerr) return fail(MOM6B_ERR_TIMEOUT, "tensor-core pipeline wait timed out");
    if (int rc = check_status(m)) return rc;
    out3[0] = acc[1] > 0.0 ? std::sqrt(acc[0] / acc[1]) : std::sqrt(acc[0]);
    out3[1] = acc[1] > 0.0 ? 1.0 : 0.0;
    out3[2] = (double)calls;
    return MOM6B_OK;
}

extern "C" int mom6b_surrogate_enable(mom6b_model* m, int on, int shadow_every, double threshold)
{
    if (!m) return fail(MOM6B_ERR_ARG, "null model");
    if (on && !m->sur) return fail(MOM6B_ERR_STATE, "no surrogate network: train or load one first");
    CK(cudaSetDevice(m->cfg.device));
    CK(cudaStreamSynchronize(m->s3d));
    if (on) {
        if (int rc = sur_buffers(m)) return rc;
        const int nc = (m->D.ie - m->D.is + 1) * (m->D.je - m->D.js + 1);
        CK(m->sur->prepare_inference(nc));   // allocations before any capture
    }
    m->sur_on = on != 0;
    m->sur_fallen = false;
    m->sur_every = shadow_every;
    m->sur_thresh = threshold;
    m->sur_steps = 0;
    invalidate_graph(m);
    return MOM6B_OK;
}

extern "C" int mom6b_surrogate_status(const mom6b_model* m, double* out10)
{
    if (!m || !out10) return fail(MOM6B_ERR_ARG, "null argument");
    const double v[10] = {m->sur_on ? 1.0 : 0.0, m->sur_fallen ? 1.0 : 0.0,
                          (double)m->sur_steps, (double)m->sur_checks,
                          (double)m->sur_fallbacks, m->sur_last_err, m->sur_max_err,
                          m->sur_loss_first, m->sur_loss_last, (double)m->sur_train_steps};
    std::memcpy(out10, v, sizeof(v));
    return MOM6B_OK;
}

// Parameters as kMlpParams floats followed by the 7 feature stds and the 2
// target stds.
extern "C" size_t mom6b_surrogate_param_count(void) { return (size_t)kMlpParams + 9; }

extern "C" int mom6b_surrogate_get_params(const mom6b_model* m, float* host, size_t n)
{
    if (!m || !host || n != mom6b_surrogate_param_count()) return fail(MOM6B_ERR_ARG, "bad argument");
    if (!m->sur) return fail(MOM6B_ERR_STATE, "no surrogate network");
    CK(cudaSetDevice(m->cfg.device));
    CK(m->sur->get_params(host));
    for (int q = 0; q < kMlpChannels; ++q) host[kMlpParams + q] = m->sur->feat_std[q];
    host[kMlpParams + 7] = m->sur->targ_std[0];
    host[kMlpParams + 8] = m->sur->targ_std[1];
    return MOM6B_OK;
}

extern "C" int mom6b_surrogate_set_params(mom6b_model* m, const float* host, size_t n)
{
    if (!m || !host || n != mom6b_surrogate_param_count()) return fail(MOM6B_ERR_ARG, "bad argument");
    CK(cudaSetDevice(m->cfg.device));
    if (!m->sur) {
        auto N = std::make_unique<Mlp>();
        CK(N->init(1024, 0, m->s3d));
        m->sur = std::move(N);
    }
    Mlp& N = *m->sur;
    for (int q = 0; q < kMlpChannels; ++q) N.feat_std[q] = host[kMlpParams + q];
    N.targ_std[0] = host[kMlpParams + 7];
    N.targ_std[1] = host[kMlpParams + 8];
    float nrm[16] = {0};
    for (int q = 0; q < kMlpChannels; ++q) nrm[q] = 1.0f / N.feat_std[q];
    nrm[7] = N.targ_std[0];
    nrm[8] = N.targ_std[1];
    CK(cudaMemcpy(N.d_norm, nrm, sizeof(nrm), cudaMemcpyHostToDevice));
    CK(N.set_params(host));
    invalidate_graph(m);
    return MOM6B_OK;
}

// ---- the network alone (tests against the CPU oracle) ------------------------
struct mom6b_mlp {
    Mlp net;
};

extern "C" int mom6b_mlp_param_count(void) { return kMlpParams; }

extern "C" int mom6b_mlp_create(int batch, uint64_t seed, mom6b_mlp** out)
{
    if (!out || batch < 128 || batch % 8) return fail(MOM6B_ERR_ARG, "bad argument");
    *out = nullptr;
    auto p = std::make_unique<mom6b_mlp>();
    CK(p->net.init(batch, seed, 0));
    *out = p.release();
    return MOM6B_OK;
}

extern "C" int mom6b_mlp_destroy(mom6b_mlp* p)
{
    delete p;
    return MOM6B_OK;
}

extern "C" int mom6b_mlp_get_params(mom6b_mlp* p, float* host, size_t n)
{
    if (!p || !host || n != (size_t)kMlpParams) return fail(MOM6B_ERR_ARG, "bad argument");
    CK(p->net.get_params(host));
    return MOM6B_OK;
}

extern "C" int mom6b_mlp_set_params(mom6b_mlp* p, const float* host, size_t n)
{
    if (!p || !host || n != (size_t)kMlpParams) return fail(MOM6B_ERR_ARG, "bad argument");
    CK(p->net.set_params(host));
    return MOM6B_OK;
}

// bf16 features [rows][176] (and optionally [176][rows]) from fp32 [rows][175].
static void mlp_pack(const float* X, int rows, std::vector<__nv_bfloat16>& row_major,
                     std::vector<__nv_bfloat16>* col_major)
{
    row_major.assign((size_t)rows * kMlpInPad, __float2bfloat16_rn(0.0f));
    if (col_major) col_major->assign((size_t)rows * kMlpInPad, __float2bfloat16_rn(0.0f));
    for (int r = 0; r < rows; ++r)
        for (int f = 0; f < kMlpIn; ++f) {
            const __nv_bfloat16 v = __float2bfloat16_rn(X[(size_t)r * kMlpIn + f]);
            row_major[(size_t)r * kMlpInPad + f] = v;
            if (col_major) (*col_major)[(size_t)f * rows + r] = v;
        }
}

static int mlp_upload(mom6b_mlp* p, const float* X, const float* Y, int B)
{
    if (B > p->net.B_cap || B < 128 || B % 8) return fail(MOM6B_ERR_ARG, "batch outside 128..capacity or not a multiple of 8");
    std::vector<__nv_bfloat16> xr, xc;
    mlp_pack(X, B, xr, &xc);
    CK(cudaMemcpy(p->net.X, xr.data(), xr.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(p->net.XT, xc.data(), xc.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(p->net.Y, Y, (size_t)B * kMlpOut * sizeof(float), cudaMemcpyHostToDevice));
    return MOM6B_OK;
}

static int mlp_check(mom6b_mlp* p)
{
    CK(cudaDeviceSynchronize());
    int e = 0;
    CK(cudaMemcpy(&e, p->net.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return fail(MOM6B_ERR_TIMEOUT, "tensor-core pipeline wait timed out");
    return MOM6B_OK;
}

extern "C" int mom6b_mlp_gradients(mom6b_mlp* p, const float* X, const float* Y, int B,
                                   float* grads, float* loss, float* out)
{
    if (!p || !X || !Y) return fail(MOM6B_ERR_ARG, "null argument");
    if (int rc = mlp_upload(p, X, Y, B)) return rc;
    CK(p->net.gradients(B, 0));
    if (int rc = mlp_check(p)) return rc;
    if (grads) CK(p->net.grads_to_host(grads, 0));
    if (loss) CK(cudaMemcpy(loss, p->net.loss, sizeof(float), cudaMemcpyDeviceToHost));
    if (out) CK(cudaMemcpy(out, p->net.out, (size_t)B * kMlpOut * sizeof(float), cudaMemcpyDeviceToHost));
    return MOM6B_OK;
}

extern "C" int mom6b_mlp_train(mom6b_mlp* p, const float* X, const float* Y, int B, float lr,
                               int nsteps, float* losses)
{
    if (!p || !X || !Y || nsteps < 0) return fail(MOM6B_ERR_ARG, "bad argument");
    if (int rc = mlp_upload(p, X, Y, B)) return rc;
    for (int t = 0; t < nsteps; ++t) {
        CK(p->net.train_step(B, lr, 0));
        if (losses) CK(cudaMemcpy(losses + t, p->net.loss, sizeof(float), cudaMemcpyDeviceToHost));
    }
    return mlp_check(p);
}

extern "C" int mom6b_mlp_predict(mom6b_mlp* p, const float* X, int n, float* out)
{
    if (!p || !X || !out || n < 1) return fail(MOM6B_ERR_ARG, "bad argument");
    CK(p->net.prepare_inference(n));
    std::vector<__nv_bfloat16> xr;
    mlp_pack(X, n, xr, nullptr);
    CK(cudaMemcpy(p->net.Xi, xr.data(), xr.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
    CK(p->net.predict(n, 0));
    if (int rc = mlp_check(p)) return rc;
    CK(cudaMemcpy(out, p->net.outi, (size_t)n * kMlpOut * sizeof(float), cudaMemcpyDeviceToHost));
    return MOM6B_OK;
}
