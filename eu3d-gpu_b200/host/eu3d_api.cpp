// eu3d_api.cpp — the C ABI (include/eu3d.h): handle lifetime, device memory,
// uploads/downloads and the per-timestep launch sequence.
#include "eu3d.h"

#include <array>
#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <tuple>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../csrc/eu3d_launch.hpp"
#include "eu3d_mech_JA919_tables.h"
#include "mlp_internal.hpp"
#include "readers.hpp"
#include "state_init.hpp"

using namespace eu3d;

struct eu_handle {
    eu_config cfg{};
    int ni = 0, nj = 0, nk = 0, bc = 0, nx = 0, ny = 0, nz = 0;
    long long n3 = 0;
    std::vector<double> x, y, z;
    MechanismTables mech;
    DevMech dmech{};
    int spec = 0; // 1 when the tables are the generated H2_JA919 ones
    bool has_mech = false, has_state = false;
    DevGrid g{};
    DevState st{};
    double *d_xyz = nullptr;
    double *d_dt = nullptr;
    unsigned long long *d_cfl_slot = nullptr; // CFL minimum of the step being set up
    double *d_time = nullptr;                 // time advanced by the CFL-driven steps of a call
    double *d_scratch = nullptr;
    double *d_inflow = nullptr; // EU_BC_ODW x-low tables ((8 + ns) planes of nj * nk)
    std::vector<void *> allocs;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t pev[4] = {nullptr, nullptr, nullptr, nullptr}; // phase boundaries (cfg.profile)
    // learned chemistry
    eu_mlp *model = nullptr;
    LearnedParams lp{};
    long long lp_capacity = 0;
    int *h_counts = nullptr; // pinned [2]
    int heavy_blocks = 0;    // persistent grid of the warp-per-cell kinetics
    // mixed precision: the timestep keeps only the FP32 primitive planes
    // current; the FP64 ones are formed on demand (k_materialize) for output
    bool prim_stale = false;
    int *d_zm_fresh = nullptr; // EU_GHOSTS_STORED's flag (eu_set_ghost_mode)
    int sms = 0;
    // one timestep captured as a CUDA graph (recaptured when what its kernels
    // take by value changes: the mechanism, the learned-chemistry settings)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_launches = 0;
    bool graph_dirty = true;
    double graph_cfl = 0;   // the CFL number the captured step sets its dt from (0: a fixed dt)
    bool graph_shared_tail = false; // captured for a batch: the stiff-fallback and deferred-cell
                                    // kinetics left to the batch's shared stage
    unsigned graph_gen = 0; // captures so far (batches rebuild when it changes)
    // launch shapes picked by eu_autotune (0: defaults)
    int flux_ci = 0, recover_block = 0, recover_minb = 0;
    // advection time scheme (eu_set_time_scheme) and the RK start-of-step state
    int time_scheme = EU_TIME_EE;
    double *d_cs0 = nullptr;
    // asynchronous output (eu_output_async): device snapshot of the fields a
    // file needs, its pinned host copy, the copy stream and the writer thread
    double *d_snap = nullptr, *h_snap = nullptr;
    size_t snap_bytes = 0;
    cudaStream_t out_stream = nullptr;
    cudaEvent_t ev_snap = nullptr, ev_host = nullptr;
    std::thread out_thread;
    eu_status out_status = EU_OK;
    std::string out_err;
    std::string err;
};

namespace {

const char *kNoHandle = "null handle";

eu_status fail(eu_handle *h, eu_status s, const char *fmt, ...)
{
    if (h) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        h->err = buf;
    }
    return s;
}

eu_status cuda_fail(eu_handle *h, cudaError_t e, const char *what)
{
    // a failed call leaves its error as the runtime's last error: clear it, so
    // the next launch's cudaGetLastError reports that launch, not this call
    (void)cudaGetLastError();
    if (e == cudaErrorMemoryAllocation)
        return fail(h, EU_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
    return fail(h, EU_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(h, call)                                                                                \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return cuda_fail((h), e_, #call);                                                      \
    } while (0)

template <typename T>
eu_status dalloc(eu_handle *h, T **p, size_t count)
{
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T));
    if (e != cudaSuccess)
        return cuda_fail(h, e, "cudaMalloc");
    h->allocs.push_back(q);
    h->bytes += count * sizeof(T);
    *p = static_cast<T *>(q);
    return EU_OK;
}

void free_all(eu_handle *h)
{
    for (void *p : h->allocs) cudaFree(p);
    h->allocs.clear();
    h->bytes = 0;
}

// DevMech from host tables; rejects sizes the kernels are not built for.
eu_status install_mechanism(eu_handle *h, const MechanismTables &m)
{
    if (m.ns <= 0 || m.nr <= 0 || m.ns > kMaxS || m.nr > kMaxR)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "mechanism sizes ns=%d nr=%d outside 1..%d / 1..%d", m.ns, m.nr,
                    kMaxS, kMaxR);
    if (!sizes_supported(m.ns, m.nr))
        return fail(h, EU_ERR_UNSUPPORTED, "no kernels built for ns=%d nr=%d (built: 9/19)", m.ns, m.nr);
    if (h->has_mech && m.ns != h->mech.ns)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "species count cannot change on a live handle");
    DevMech d;
    std::memset(&d, 0, sizeof d);
    d.ns = m.ns;
    d.nr = m.nr;
    int nu_int = 1;
    for (int s = 0; s < m.ns; ++s) {
        if (!(m.mw[s] > 0))
            return fail(h, EU_ERR_INVALID_ARGUMENT, "molecular weight of species %d not positive", s);
        d.mw[s] = m.mw[s];
        d.ri[s] = kRUniv / m.mw[s];
        for (int k = 0; k < 9; ++k) {
            d.clo[k][s] = m.coeff_lo[k * m.ns + s];
            d.chi[k][s] = m.coeff_hi[k * m.ns + s];
        }
    }
    for (int r = 0; r < m.nr; ++r) {
        d.af[r] = m.af[r];
        d.bf[r] = m.bf[r];
        d.eaf[r] = m.eaf[r];
        double xr = 0;
        int tb = 0;
        for (int s = 0; s < m.ns; ++s) {
            const double f = m.stoi_f[s * m.nr + r], b = m.stoi_b[s * m.nr + r];
            d.sf[r][s] = f;
            d.sb[r][s] = b;
            d.tb[r][s] = m.tb[s * m.nr + r];
            xr += (b - f);
            if (m.tb[s * m.nr + r] != 0)
                tb = 1;
            for (double v : {f, b})
                if (!(v == 0.0 || v == 1.0 || v == 2.0))
                    nu_int = 0;
        }
        d.xr[r] = xr;
        d.has_tb[r] = tb;
    }
    if (!nu_int)
        return fail(h, EU_ERR_UNSUPPORTED, "stoichiometric coefficients other than 0, 1, 2 are not supported");
    d.nu_int = nu_int;
    const bool first = !h->has_mech;
    h->spec = matches_JA919(m.ns, m.nr, m.mw.data(), m.coeff_lo.data(), m.coeff_hi.data(), m.af.data(), m.bf.data(),
                            m.eaf.data(), m.stoi_f.data(), m.stoi_b.data(), m.tb.data())
                  ? 1
                  : 0;
    h->mech = m;
    h->dmech = d;
    h->has_mech = true;
    h->graph_dirty = true; // the kernels take the tables by value
    if (!first)
        return EU_OK;

    // State buffers depend on ns: allocate them with the first mechanism.
    const long long n3 = h->n3;
    const int ns = m.ns;
    eu_status s;
    if ((s = dalloc(h, &h->st.prim, size_t(7 + ns) * n3)) != EU_OK) return s;
    if (h->cfg.precision == EU_PREC_MIXED)
        if ((s = dalloc(h, &h->st.prim32, size_t(7 + ns) * n3)) != EU_OK) return s;
    if ((s = dalloc(h, &h->st.cs, size_t(ns + 4) * n3)) != EU_OK) return s;
    if ((s = dalloc(h, &h->st.T, size_t(n3))) != EU_OK) return s;
    if ((s = dalloc(h, &h->st.E, size_t(n3))) != EU_OK) return s;
    if ((s = dalloc(h, &h->st.nchem, size_t(n3))) != EU_OK) return s;
    if (h->cfg.record_sources)
        if ((s = dalloc(h, &h->st.cms, size_t(ns) * n3)) != EU_OK) return s;
    if ((s = dalloc(h, &h->st.counters, size_t(kCntCount))) != EU_OK) return s;
    if ((s = dalloc(h, &h->d_scratch, size_t(n3))) != EU_OK) return s;
    if (h->cfg.precision == EU_PREC_MIXED) {
        if ((s = dalloc(h, &h->st.heavy, size_t(2) + size_t(h->ni) * h->nj * h->nk)) != EU_OK) return s;
        CK(h, cudaMemsetAsync(h->st.heavy, 0, 2 * sizeof(int), h->stream));
    }
    CK(h, cudaMemsetAsync(h->st.prim, 0, size_t(7 + ns) * n3 * sizeof(double), h->stream));
    if (h->st.prim32)
        CK(h, cudaMemsetAsync(h->st.prim32, 0, size_t(7 + ns) * n3 * sizeof(float), h->stream));
    CK(h, cudaMemsetAsync(h->st.cs, 0, size_t(ns + 4) * n3 * sizeof(double), h->stream));
    CK(h, cudaMemsetAsync(h->st.T, 0, size_t(n3) * sizeof(double), h->stream));
    CK(h, cudaMemsetAsync(h->st.E, 0, size_t(n3) * sizeof(double), h->stream));
    CK(h, cudaMemsetAsync(h->st.nchem, 0, size_t(n3) * sizeof(int), h->stream));
    if (h->st.cms)
        CK(h, cudaMemsetAsync(h->st.cms, 0, size_t(ns) * n3 * sizeof(double), h->stream));
    CK(h, cudaMemsetAsync(h->st.counters, 0, kCntCount * sizeof(unsigned long long), h->stream));
    return EU_OK;
}

LaunchArgs launch_args(eu_handle *h)
{
    LaunchArgs a;
    a.mech = &h->dmech;
    a.g = h->g;
    a.st = h->st;
    a.dt_dev = h->d_dt;
    a.max_substeps = h->cfg.max_substeps > 0 ? h->cfg.max_substeps : (1 << 20);
    a.precision = h->cfg.precision;
    a.chemistry = h->cfg.chemistry;
    a.spec = h->spec;
    a.sms = h->sms;
    a.flux_ci = h->flux_ci;
    a.recover_block = h->recover_block;
    a.recover_minb = h->recover_minb;
    a.stream = h->stream;
    return a;
}

using TuneKey = std::tuple<int, int, int, int, int, int, int>;
std::mutex g_tune_mutex;                            // guards g_tuned
std::map<TuneKey, std::array<int, 3>> g_tuned;      // (flux_ci, recover_block, recover_minb) per grid and mode

TuneKey tune_key(const eu_handle *h)
{
    return TuneKey(h->ni, h->nj, h->nk, h->cfg.precision, h->cfg.arith, h->cfg.chemistry, h->cfg.device);
}

void drop_graph(eu_handle *h)
{
    if (h->graph_exec)
        cudaGraphExecDestroy(h->graph_exec);
    if (h->graph)
        cudaGraphDestroy(h->graph);
    h->graph_exec = nullptr;
    h->graph = nullptr;
    h->graph_dirty = true;
}

bool is_strict(const eu_handle *h) { return h->cfg.arith == EU_ARITH_STRICT; }

// Kernels of the handle's flavour: mixed precision has its own translation
// unit (FP32 fluxes, fast FP64 forms) whatever cfg.arith says; FP64 follows
// cfg.arith.
const Launchers &flavour(const eu_handle *h)
{
    if (h->cfg.precision == EU_PREC_MIXED)
        return mixed::launchers;
    return is_strict(h) ? strict::launchers : fast::launchers;
}


} // namespace

namespace eu3d {
bool sizes_supported(int ns, int nr) { return ns == 9 && nr == 19; }
} // namespace eu3d

extern "C" {

int eu_abi_version(void) { return EU3D_ABI_VERSION; }

eu_status eu_read_value(const char *path, const char *key, double *value)
{
    if (!path || !key || !value)
        return EU_ERR_INVALID_ARGUMENT;
    KeyValueFile f;
    if (!f.read(path))
        return EU_ERR_IO;
    if (!f.has(key))
        return EU_ERR_INVALID_ARGUMENT;
    *value = f.get_double(key);
    return EU_OK;
}

eu_status eu_read_grid(const char *grid_path, eu_config *cfg)
{
    if (!grid_path || !cfg)
        return EU_ERR_INVALID_ARGUMENT;
    GridSpec g;
    std::string err;
    if (!read_grid(grid_path, g, err))
        return EU_ERR_IO;
    cfg->total_ni = g.total_ni;
    cfg->total_nj = g.total_nj;
    cfg->total_nk = g.total_nk;
    cfg->xa = g.xa;
    cfg->xb = g.xb;
    cfg->ya = g.ya;
    cfg->yb = g.yb;
    cfg->za = g.za;
    cfg->zb = g.zb;
    cfg->bc = g.bc;
    return EU_OK;
}

namespace {
MechanismTables tables_from(const eu_mechanism *mm)
{
    MechanismTables m;
    m.ns = mm->ns;
    m.nr = mm->nr;
    const int ns = m.ns, nr = m.nr;
    m.mw.assign(mm->mw, mm->mw + ns);
    m.coeff_lo.assign(mm->coeff_lo, mm->coeff_lo + 9 * ns);
    m.coeff_hi.assign(mm->coeff_hi, mm->coeff_hi + 9 * ns);
    m.af.assign(mm->af, mm->af + nr);
    m.bf.assign(mm->bf, mm->bf + nr);
    m.eaf.assign(mm->eaf, mm->eaf + nr);
    m.stoi_f.assign(mm->stoi_f, mm->stoi_f + ns * nr);
    m.stoi_b.assign(mm->stoi_b, mm->stoi_b + ns * nr);
    m.tb.assign(mm->tb, mm->tb + ns * nr);
    return m;
}

bool mechanism_complete(const eu_mechanism *mm)
{
    return mm && mm->mw && mm->coeff_lo && mm->coeff_hi && mm->af && mm->bf && mm->eaf && mm->stoi_f &&
           mm->stoi_b && mm->tb && mm->ns > 0 && mm->nr > 0 && mm->ns <= kMaxS && mm->nr <= kMaxR;
}
} // namespace

eu_status eu_parse_mechanism(const char *mech_path, const char *thermo_path, int *ns, int *nr, double *mw,
                             double *coeff_lo, double *coeff_hi, double *af, double *bf, double *eaf,
                             double *stoi_f, double *stoi_b, double *tb)
{
    if (!mech_path || !thermo_path)
        return EU_ERR_INVALID_ARGUMENT;
    MechanismTables m;
    std::string err;
    if (!read_mechanism(mech_path, thermo_path, m, err))
        return EU_ERR_IO;
    if (ns) *ns = m.ns;
    if (nr) *nr = m.nr;
    auto cp = [](double *dst, const std::vector<double> &v) {
        if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(double));
    };
    cp(mw, m.mw);
    cp(coeff_lo, m.coeff_lo);
    cp(coeff_hi, m.coeff_hi);
    cp(af, m.af);
    cp(bf, m.bf);
    cp(eaf, m.eaf);
    cp(stoi_f, m.stoi_f);
    cp(stoi_b, m.stoi_b);
    cp(tb, m.tb);
    return EU_OK;
}

eu_status eu_initial_state(const eu_mechanism *mm, int ni, int nj, int nk, int bc, const double *P, const double *T,
                           const double *U, const double *V, const double *W, const double *Y, double *prim,
                           double *cs, double *T_out, double *E_out)
{
    if (!mechanism_complete(mm) || !P || !T || !U || !V || !W || !Y || !prim || !cs || !T_out || !E_out || bc < 1 ||
        ni < 2 || nj < 2 || nk < 2)
        return EU_ERR_INVALID_ARGUMENT;
    const MechanismTables m = tables_from(mm);
    std::vector<double> pv, cv, tv, ev;
    primitive_to_state(m, ni, nj, nk, bc, P, T, U, V, W, Y, pv, cv, tv, ev);
    std::memcpy(prim, pv.data(), pv.size() * sizeof(double));
    std::memcpy(cs, cv.data(), cv.size() * sizeof(double));
    std::memcpy(T_out, tv.data(), tv.size() * sizeof(double));
    std::memcpy(E_out, ev.data(), ev.size() * sizeof(double));
    return EU_OK;
}

eu_status eu_create(const eu_config *cfg, eu_handle **out)
{
    if (!cfg || !out)
        return EU_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (cfg->bc != 2 || cfg->total_ni < 2 || cfg->total_nj < 2 || cfg->total_nk < 2)
        return EU_ERR_INVALID_ARGUMENT;
    if (cfg->precision != EU_PREC_FP64 && cfg->precision != EU_PREC_MIXED)
        return EU_ERR_INVALID_ARGUMENT;
    if (cfg->chemistry != EU_CHEM_STIFF && cfg->chemistry != EU_CHEM_FROZEN && cfg->chemistry != EU_CHEM_LEARNED)
        return EU_ERR_INVALID_ARGUMENT;
    if (cfg->boundary != EU_BC_RSBI && cfg->boundary != EU_BC_ZND && cfg->boundary != EU_BC_ODW)
        return EU_ERR_INVALID_ARGUMENT;
    // x blocks: the reference's layout rule (src/Mesh.cpp:64-75) and at least
    // bc + 2 nodes per block (a message reaches node 2 bc)
    const int blocks_x = cfg->blocks_x > 1 ? cfg->blocks_x : 1;
    if (blocks_x > 1 && ((cfg->total_ni - 1) % blocks_x != 0 || cfg->block_x < 0 || cfg->block_x >= blocks_x ||
                         (cfg->total_ni - 1) / blocks_x + 1 < 2 * cfg->bc + 1))
        return EU_ERR_INVALID_ARGUMENT;
    if (blocks_x == 1 && cfg->block_x != 0)
        return EU_ERR_INVALID_ARGUMENT;
    // the kernels' flat node indices stay below 2^31
    if ((long long)((cfg->total_ni - 1) / blocks_x + 1 + 4) * (cfg->total_nj + 4) * (cfg->total_nk + 4) >= (1LL << 31))
        return EU_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return EU_ERR_CUDA;
    if (cfg->device < 0 || cfg->device >= ndev)
        return EU_ERR_INVALID_ARGUMENT;
    eu_handle *h = new (std::nothrow) eu_handle;
    if (!h)
        return EU_ERR_OUT_OF_MEMORY;
    h->cfg = *cfg;
    if (cudaSetDevice(cfg->device) != cudaSuccess) {
        delete h;
        return EU_ERR_CUDA;
    }
    h->ni = (cfg->total_ni - 1) / blocks_x + 1;
    h->nj = cfg->total_nj;
    h->nk = cfg->total_nk;
    h->bc = cfg->bc;
    h->nx = h->ni + 2 * h->bc;
    h->ny = h->nj + 2 * h->bc;
    h->nz = h->nk + 2 * h->bc;
    h->n3 = (long long)h->nx * h->ny * h->nz;
    h->x = node_coordinates(cfg->total_ni, cfg->xa, cfg->xb, h->bc, blocks_x, cfg->block_x);
    h->y = node_coordinates(h->nj, cfg->ya, cfg->yb, h->bc);
    h->z = node_coordinates(h->nk, cfg->za, cfg->zb, h->bc);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess) {
        eu_destroy(h);
        return EU_ERR_CUDA;
    }
    for (auto &e : h->pev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            eu_destroy(h);
            return EU_ERR_CUDA;
        }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cfg->device) != cudaSuccess || sms < 1)
        sms = 1;
    h->heavy_blocks = 3 * sms; // 3 blocks of 4 warps per SM (its register target), each warp a cell at a time
    h->sms = sms;
    eu_status s;
    if ((s = dalloc(h, &h->d_xyz, size_t(h->nx + h->ny + h->nz))) != EU_OK ||
        (s = dalloc(h, &h->d_dt, size_t(1))) != EU_OK || (s = dalloc(h, &h->d_time, size_t(1))) != EU_OK ||
        (s = dalloc(h, &h->d_cfl_slot, size_t(1))) != EU_OK) {
        eu_destroy(h);
        return s;
    }
    {
        const unsigned long long inf_bits = 0x7ff0000000000000ULL; // +inf: no minimum yet
        if (cudaMemcpy(h->d_cfl_slot, &inf_bits, sizeof inf_bits, cudaMemcpyHostToDevice) != cudaSuccess) {
            eu_destroy(h);
            return EU_ERR_CUDA;
        }
    }
    std::vector<double> xyz;
    xyz.insert(xyz.end(), h->x.begin(), h->x.end());
    xyz.insert(xyz.end(), h->y.begin(), h->y.end());
    xyz.insert(xyz.end(), h->z.begin(), h->z.end());
    if (cudaMemcpy(h->d_xyz, xyz.data(), xyz.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        eu_destroy(h);
        return EU_ERR_CUDA;
    }
    h->g.ni = h->ni;
    h->g.nj = h->nj;
    h->g.nk = h->nk;
    h->g.bc = h->bc;
    h->g.nx = h->nx;
    h->g.ny = h->ny;
    h->g.nz = h->nz;
    h->g.n3 = h->n3;
    h->g.x = h->d_xyz;
    h->g.y = h->d_xyz + h->nx;
    h->g.z = h->d_xyz + h->nx + h->ny;
    h->g.d_nk = make_fastdiv(unsigned(h->nk));
    h->g.d_njnk = make_fastdiv(unsigned(h->nj) * unsigned(h->nk));
    h->g.d_nink = make_fastdiv(unsigned(h->ni) * unsigned(h->nk));
    h->g.d_ghost = make_fastdiv(unsigned(2 * h->bc));
    h->g.d_ghost_nj = make_fastdiv(unsigned(2 * h->bc) * unsigned(h->nj));
    h->g.d_nz = make_fastdiv(unsigned(h->nz));
    h->g.d_nynz = make_fastdiv(unsigned(h->ny) * unsigned(h->nz));
    h->g.bc_kind = cfg->boundary;
    h->g.exch_lo = blocks_x > 1 && cfg->block_x > 0;
    h->g.exch_hi = blocks_x > 1 && cfg->block_x < blocks_x - 1;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tuned.find(tune_key(h));
        if (it != g_tuned.end()) {
            h->flux_ci = it->second[0];
            h->recover_block = it->second[1];
            h->recover_minb = it->second[2];
        }
    }
    *out = h;
    return EU_OK;
}

eu_status eu_destroy(eu_handle *h)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->cfg.device);
    if (h->out_thread.joinable())
        h->out_thread.join();
    if (h->stream)
        cudaStreamSynchronize(h->stream);
    drop_graph(h);
    free_all(h);
    if (h->d_snap) cudaFree(h->d_snap);
    if (h->h_snap) cudaFreeHost(h->h_snap);
    if (h->ev_snap) cudaEventDestroy(h->ev_snap);
    if (h->ev_host) cudaEventDestroy(h->ev_host);
    if (h->out_stream) cudaStreamDestroy(h->out_stream);
    if (h->h_counts)
        cudaFreeHost(h->h_counts);
    for (auto &e : h->pev)
        if (e) cudaEventDestroy(e);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return EU_OK;
}

const char *eu_last_error(const eu_handle *h) { return h ? h->err.c_str() : kNoHandle; }

eu_status eu_load_mechanism(eu_handle *h, const char *mech_path, const char *thermo_path)
{
    if (!h || !mech_path || !thermo_path)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(h->cfg.device);
    MechanismTables m;
    std::string err;
    if (!read_mechanism(mech_path, thermo_path, m, err))
        return fail(h, EU_ERR_IO, "%s", err.c_str());
    return install_mechanism(h, m);
}

eu_status eu_set_mechanism(eu_handle *h, const eu_mechanism *mm)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!mechanism_complete(mm))
        return fail(h, EU_ERR_INVALID_ARGUMENT, "null table or sizes out of range");
    cudaSetDevice(h->cfg.device);
    return install_mechanism(h, tables_from(mm));
}

eu_status eu_get_mechanism(const eu_handle *h, int *ns, int *nr, double *mw, double *coeff_lo, double *coeff_hi,
                           double *af, double *bf, double *eaf, double *stoi_f, double *stoi_b, double *tb)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!h->has_mech)
        return EU_ERR_NOT_READY;
    const MechanismTables &m = h->mech;
    if (ns) *ns = m.ns;
    if (nr) *nr = m.nr;
    auto cp = [](double *dst, const std::vector<double> &v) {
        if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(double));
    };
    cp(mw, m.mw);
    cp(coeff_lo, m.coeff_lo);
    cp(coeff_hi, m.coeff_hi);
    cp(af, m.af);
    cp(bf, m.bf);
    cp(eaf, m.eaf);
    cp(stoi_f, m.stoi_f);
    cp(stoi_b, m.stoi_b);
    cp(tb, m.tb);
    return EU_OK;
}

eu_status eu_node_coordinates(const eu_handle *h, double *x, double *y, double *z)
{
    if (!h || !x || !y || !z)
        return EU_ERR_INVALID_ARGUMENT;
    std::memcpy(x, h->x.data(), h->x.size() * sizeof(double));
    std::memcpy(y, h->y.data(), h->y.size() * sizeof(double));
    std::memcpy(z, h->z.data(), h->z.size() * sizeof(double));
    return EU_OK;
}

eu_status eu_set_state(eu_handle *h, const double *cs, const double *T, const double *E, const double *P,
                       const double *D, const double *U, const double *V, const double *W, const double *H,
                       const double *G, const double *Y)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!cs || !T || !E || !P || !D || !U || !V || !W || !H || !G || !Y)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "null argument");
    if (!h->has_mech)
        return fail(h, EU_ERR_NOT_READY, "load a mechanism first");
    cudaSetDevice(h->cfg.device);
    const long long n3 = h->n3;
    const int ns = h->mech.ns;
    const size_t b = size_t(n3) * sizeof(double);
    const double *planes[7] = {P, D, U, V, W, H, G};
    for (int f = 0; f < 7; ++f) CK(h, cudaMemcpyAsync(h->st.prim + f * n3, planes[f], b, cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemcpyAsync(h->st.prim + 7 * n3, Y, ns * b, cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemcpyAsync(h->st.cs, cs, (ns + 4) * b, cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemcpyAsync(h->st.T, T, b, cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemcpyAsync(h->st.E, E, b, cudaMemcpyHostToDevice, h->stream));
    if (h->st.prim32) // the FP32 planes the mixed-precision fluxes read, converted on the device
        CK(h, strict::launch_to_f32(h->st.prim, h->st.prim32, (long long)(7 + ns) * n3, h->stream));
    if (h->st.zm_fresh) // EU_GHOSTS_STORED: the uploaded ghosts are the caller's; the next fill forms the z faces
        CK(h, cudaMemsetAsync(h->st.zm_fresh, 0, sizeof(int), h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    h->has_state = true;
    h->prim_stale = false;
    return EU_OK;
}

eu_status eu_set_conserved(eu_handle *h, const double *cs, const double *T, const double *E)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!cs || !T || !E)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "null argument");
    if (!h->has_mech)
        return fail(h, EU_ERR_NOT_READY, "load a mechanism first");
    cudaSetDevice(h->cfg.device);
    const long long n3 = h->n3;
    const size_t b = size_t(n3) * sizeof(double);
    CK(h, cudaMemcpyAsync(h->st.cs, cs, (h->mech.ns + 4) * b, cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemcpyAsync(h->st.T, T, b, cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemcpyAsync(h->st.E, E, b, cudaMemcpyHostToDevice, h->stream));
    // Update_after_CS on the interior nodes (the recovery of the step, no kinetics)
    CK(h, flavour(h).recover_react(launch_args(h), false));
    CK(h, cudaStreamSynchronize(h->stream));
    h->has_state = true;
    h->prim_stale = h->st.prim32 != nullptr; // mixed precision: the FP64 planes are formed on demand
    return EU_OK;
}

eu_status eu_set_primitive(eu_handle *h, const double *P, const double *T, const double *U, const double *V,
                           const double *W, const double *Y)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!P || !T || !U || !V || !W || !Y)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "null argument");
    if (!h->has_mech)
        return fail(h, EU_ERR_NOT_READY, "load a mechanism first");
    std::vector<double> prim, cs, Tv, Ev;
    primitive_to_state(h->mech, h->ni, h->nj, h->nk, h->bc, P, T, U, V, W, Y, prim, cs, Tv, Ev);
    const long long n3 = h->n3;
    return eu_set_state(h, cs.data(), Tv.data(), Ev.data(), &prim[0], &prim[n3], &prim[2 * n3], &prim[3 * n3],
                        &prim[4 * n3], &prim[5 * n3], &prim[6 * n3], &prim[7 * n3]);
}

eu_status eu_set_inflow(eu_handle *h, const double *P, const double *T, const double *U, const double *V,
                        const double *W, const double *Y)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!P || !T || !U || !V || !W || !Y)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "null argument");
    if (!h->has_mech)
        return fail(h, EU_ERR_NOT_READY, "load a mechanism first");
    // the (j, k) tables as a one-plane grid without ghosts: FieldInitial's
    // derived values on every node
    std::vector<double> prim, cs, Tv, Ev;
    primitive_to_state(h->mech, 1, h->nj, h->nk, 0, P, T, U, V, W, Y, prim, cs, Tv, Ev);
    const size_t nt = size_t(h->nj) * h->nk, nf = 7 + size_t(h->mech.ns);
    prim.insert(prim.end(), Tv.begin(), Tv.end()); // T after the primitive planes
    cudaSetDevice(h->cfg.device);
    if (!h->d_inflow) {
        eu_status st = dalloc(h, &h->d_inflow, (nf + 1) * nt);
        if (st != EU_OK)
            return st;
    }
    CK(h, cudaMemcpyAsync(h->d_inflow, prim.data(), (nf + 1) * nt * sizeof(double), cudaMemcpyHostToDevice,
                          h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    h->st.inflow = h->d_inflow;
    h->graph_dirty = true;
    return EU_OK;
}

eu_status eu_set_time_scheme(eu_handle *h, int scheme)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (scheme != EU_TIME_EE && scheme != EU_TIME_RK3)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "unknown time scheme %d", scheme);
    if (!h->has_mech)
        return fail(h, EU_ERR_NOT_READY, "load a mechanism first");
    if (scheme == EU_TIME_RK3 && !h->d_cs0) {
        cudaSetDevice(h->cfg.device);
        eu_status st = dalloc(h, &h->d_cs0, size_t(h->n3) * (h->mech.ns + 4));
        if (st != EU_OK)
            return st;
    }
    h->time_scheme = scheme;
    h->graph_dirty = true;
    return EU_OK;
}

eu_status eu_set_ghost_mode(eu_handle *h, int mode)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (mode != EU_GHOSTS_REFERENCE && mode != EU_GHOSTS_STORED)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "unknown ghost mode %d", mode);
    if (!h->has_mech)
        return fail(h, EU_ERR_NOT_READY, "load a mechanism first");
    if (mode == EU_GHOSTS_STORED && (h->g.bc_kind == EU_BC_ODW || h->nk < h->bc))
        // the ODW fill rebuilds the z ghosts' thermo; with fewer than bc
        // interior z nodes a z ghost mirrors another ghost
        return fail(h, EU_ERR_INVALID_ARGUMENT, "stored z ghosts need the RSBI or ZND fill and nk >= %d", h->bc);
    cudaSetDevice(h->cfg.device);
    if (mode == EU_GHOSTS_STORED) {
        if (!h->d_zm_fresh) {
            eu_status st = dalloc(h, &h->d_zm_fresh, size_t(1));
            if (st != EU_OK)
                return st;
        }
        // the ghosts as they stand are the ghost fill's: the next fill forms the z faces
        CK(h, cudaMemsetAsync(h->d_zm_fresh, 0, sizeof(int), h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        h->st.zm_fresh = h->d_zm_fresh;
        h->st.zm_dnz = make_fastdiv(unsigned(h->nz));
        h->st.zm_nz = int(h->nz);
        h->st.zm_nk = h->nk;
        h->st.zm_bc = h->bc;
    } else {
        h->st.zm_fresh = nullptr;
    }
    h->graph_dirty = true; // the kernels take the state by value
    return EU_OK;
}

eu_status eu_set_odw_wall(eu_handle *h, int first_wall_node)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (h->cfg.boundary != EU_BC_ODW)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "the wall start applies to EU_BC_ODW handles");
    if (first_wall_node < 0 || first_wall_node > h->cfg.total_ni)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "first wall node %d outside 0 .. %d", first_wall_node,
                    h->cfg.total_ni);
    // this block's local index of that global node (x blocks share one node)
    const int first = (h->cfg.blocks_x > 1 ? h->cfg.block_x : 0) * (h->ni - 1);
    int local = first_wall_node - first;
    local = local < 0 ? 0 : (local > h->ni ? h->ni : local);
    if (local > 0 && !h->st.inflow)
        return fail(h, EU_ERR_NOT_READY, "set the freestream tables (eu_set_inflow) first");
    h->g.wall_i0 = local;
    h->graph_dirty = true;
    return EU_OK;
}

namespace {

// Atoms of each element in a species name such as "H2O2" or "AR".
bool element_counts(const std::string &name, double (&cnt)[6])
{
    static const char *sym[6] = {"H", "O", "N", "C", "AR", "HE"};
    for (double &c : cnt) c = 0;
    size_t i = 0;
    std::string up;
    for (char ch : name) up += char(std::toupper((unsigned char)ch));
    while (i < up.size()) {
        int e = -1;
        if (up.compare(i, 2, "AR") == 0) e = 4;
        else if (up.compare(i, 2, "HE") == 0) e = 5;
        else if (up[i] == 'H') e = 0;
        else if (up[i] == 'O') e = 1;
        else if (up[i] == 'N') e = 2;
        else if (up[i] == 'C') e = 3;
        if (e < 0)
            return false;
        i += std::strlen(sym[e]);
        int n = 0;
        while (i < up.size() && std::isdigit((unsigned char)up[i])) n = n * 10 + (up[i++] - '0');
        cnt[e] += n ? n : 1;
    }
    return true;
}

// P = I - A^T (A A^T)^-1 A with A[e][s] the mass fraction of element e in
// species s: the closest change (in the Euclidean sense) that conserves every
// element's mass, which also conserves sum Y. Without species names the
// projector only removes the mean (sum Y conserved).
void element_projector(const MechanismTables &m, double (&P)[kMaxS][kMaxS])
{
    static const double aw[6] = {1.00794, 15.9994, 14.0067, 12.011, 39.948, 4.002602};
    const int ns = m.ns;
    std::vector<std::vector<double>> A;
    bool named = (int)m.species.size() >= ns;
    std::vector<std::array<double, 6>> cnt(ns);
    for (int s = 0; named && s < ns; ++s) {
        double c[6];
        named = element_counts(m.species[s], c);
        for (int e = 0; e < 6; ++e) cnt[s][e] = c[e];
    }
    if (named) {
        for (int e = 0; e < 6; ++e) {
            std::vector<double> row(ns, 0.0);
            bool any = false;
            for (int s = 0; s < ns; ++s) {
                row[s] = cnt[s][e] * aw[e] / m.mw[s];
                any |= row[s] != 0;
            }
            if (any)
                A.push_back(row);
        }
    } else {
        A.push_back(std::vector<double>(ns, 1.0));
    }
    const int ne = (int)A.size();
    // G = A A^T, solve G X = A for X (ne x ns), P = I - A^T X
    std::vector<std::vector<double>> G(ne, std::vector<double>(ne, 0.0)), X = A;
    for (int a = 0; a < ne; ++a)
        for (int b = 0; b < ne; ++b)
            for (int s = 0; s < ns; ++s) G[a][b] += A[a][s] * A[b][s];
    for (int c = 0; c < ne; ++c) { // Gauss-Jordan with partial pivoting
        int piv = c;
        for (int r = c + 1; r < ne; ++r)
            if (std::fabs(G[r][c]) > std::fabs(G[piv][c])) piv = r;
        std::swap(G[c], G[piv]);
        std::swap(X[c], X[piv]);
        const double d = G[c][c];
        for (int k = 0; k < ne; ++k) G[c][k] /= d;
        for (int s = 0; s < ns; ++s) X[c][s] /= d;
        for (int r = 0; r < ne; ++r)
            if (r != c) {
                const double f = G[r][c];
                for (int k = 0; k < ne; ++k) G[r][k] -= f * G[c][k];
                for (int s = 0; s < ns; ++s) X[r][s] -= f * X[c][s];
            }
    }
    for (int i = 0; i < kMaxS; ++i)
        for (int j = 0; j < kMaxS; ++j) P[i][j] = 0.0;
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j < ns; ++j) {
            double v = (i == j) ? 1.0 : 0.0;
            for (int e = 0; e < ne; ++e) v -= A[e][i] * X[e][j];
            P[i][j] = v;
        }
}

// One learned-chemistry phase of a step: recover + classify every cell,
// features of the queued cells, the ensemble, gate + apply, stiff fallback.
// The queue kernels read the queue lengths on the device; with the model's
// fused inference kernel nothing here waits on the host, so the phase can be
// captured in the step's graph. Otherwise (a model shape without the fused
// kernel) the queue length is read back to size the layer-wise GEMMs.
eu_status learned_chemistry(eu_handle *h, const LaunchArgs &a, const Launchers &L, int *launches, bool fallback)
{
    LearnedParams lp = h->lp;
    const int ns = h->mech.ns;
    CK(h, cudaMemsetAsync(lp.counts, 0, 5 * sizeof(int), h->stream));
    // recovery appends the active cells to lp.active (length counts[3]); the
    // routing sends the ones needing few substeps to the stiff kinetics and
    // the rest to the model's queue (lp.queue, length counts[0])
    LearnedParams lpa = lp;
    lpa.queue = lp.active;
    lpa.counts = lp.counts + 3;
    CK(h, L.recover_classify(a, lpa));
    CK(h, L.learned_route(a, lp));
    CK(h, L.learned_features(a, lp));
    *launches += 3;
    if (mlp_has_fused(h->model)) {
        lp.pred_row = (long long)lp.members * (ns + 1);
        lp.pred_mem = ns + 1;
        eu_status s = mlp_predict_queue(h->model, lp.feat, lp.counts, int(h->lp_capacity), lp.pred, lp.pred_row,
                                        lp.pred_mem, h->stream);
        if (s != EU_OK)
            return fail(h, s, "learned model: %s", eu_mlp_last_error(h->model));
        ++*launches;
    } else {
        CK(h, cudaMemcpyAsync(h->h_counts, lp.counts, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        const int nq = h->h_counts[0];
        lp.pred_row = ns + 1;
        lp.pred_mem = (long long)nq * (ns + 1);
        if (nq > 0) {
            eu_status s = mlp_predict_stream(h->model, lp.feat, nq, lp.pred, h->stream);
            if (s != EU_OK)
                return fail(h, s, "learned model: %s", eu_mlp_last_error(h->model));
            // per batch of rows: packing, then the layers and the unscaling of every member
            *launches += mlp_batches(h->model, nq) * (1 + lp.members * (mlp_layers(h->model) + 1));
        }
    }
    CK(h, L.learned_apply(a, lp));
    ++*launches;
    if (fallback) {
        CK(h, L.react_queue(a, lp.fallback, lp.counts + 1, kCntFallback));
        ++*launches;
    }
    return EU_OK;
}

// The launches of one timestep on h->stream (run eagerly or recorded into the
// step's graph). phase (profile mode) receives per-phase event times.
// shared_tail: leave the stiff-fallback queue and the deferred cells to a
// batch's shared kinetics stage (their queues are filled, not drained).
eu_status step_launches(eu_handle *h, const LaunchArgs &a, const Launchers &L, bool prof, int *launches,
                        double cfl = 0, bool shared_tail = false)
{
    const bool react = h->cfg.chemistry == EU_CHEM_STIFF;
    const bool learned = h->cfg.chemistry == EU_CHEM_LEARNED;
    if (cfl > 0) { // this step's dt from the current state (Flowfield::CFLcondition)
        CK(h, strict::launch_cfl(a, cfl, h->d_cfl_slot, h->d_time));
        *launches += 2;
    }
    CK(h, cudaMemsetAsync(h->st.counters, 0, kCntPerStep * sizeof(unsigned long long), h->stream));
    if (prof) CK(h, cudaEventRecord(h->pev[0], h->stream));
    if (h->time_scheme == EU_TIME_RK3) {
        // three-stage TVD Runge-Kutta advection (Shu-Osher): each stage its ghost
        // fill, flux divergence (CS += dt L), combination with the start-of-step
        // state and recovery; the chemistry phase below recovers the last stage.
        // Profile phases: ghost fill = the first stage's, flux = the rest of
        // the advection.
        const size_t cs_bytes = size_t(h->n3) * (h->mech.ns + 4) * sizeof(double);
        CK(h, cudaMemcpyAsync(h->d_cs0, h->st.cs, cs_bytes, cudaMemcpyDeviceToDevice, h->stream));
        static const double ca[3] = {0.0, 0.75, 1.0 / 3.0}, cb[3] = {1.0, 0.25, 2.0 / 3.0};
        for (int q = 0; q < 3; ++q) {
            CK(h, L.boundary(a));
            if (prof && q == 0) CK(h, cudaEventRecord(h->pev[1], h->stream));
            CK(h, L.flux_update(a));
            *launches += 2;
            if (q > 0) {
                // explicitly rounded products and sum: the same in every flavour
                CK(h, strict::launch_rk_combine(a, h->d_cs0, ca[q], cb[q]));
                ++*launches;
            }
            if (q < 2) {
                CK(h, L.recover_react(a, false));
                ++*launches;
            }
        }
        if (prof) CK(h, cudaEventRecord(h->pev[2], h->stream));
    } else {
        CK(h, L.boundary(a));
        if (prof) CK(h, cudaEventRecord(h->pev[1], h->stream));
        CK(h, L.flux_update(a));
        if (prof) CK(h, cudaEventRecord(h->pev[2], h->stream));
        *launches += 2;
    }
    const bool heavy = h->st.heavy && (learned || react);
    if (heavy)
        CK(h, cudaMemsetAsync(h->st.heavy, 0, 2 * sizeof(int), h->stream));
    if (learned) {
        eu_status ls = learned_chemistry(h, a, L, launches, !shared_tail);
        if (ls != EU_OK)
            return ls;
    } else {
        CK(h, L.recover_react(a, react));
        ++*launches;
    }
    if (heavy && !shared_tail) { // warp-per-cell kinetics of the cells deferred above
        CK(h, L.react_heavy(a, h->heavy_blocks));
        ++*launches;
    }
    if (prof)
        CK(h, cudaEventRecord(h->pev[3], h->stream));
    return EU_OK;
}

// Records one timestep into h->graph and instantiates it.
eu_status capture_step(eu_handle *h, const LaunchArgs &a, const Launchers &L, double cfl = 0,
                       bool shared_tail = false)
{
    drop_graph(h);
    int launches = 0;
    CK(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    eu_status s = step_launches(h, a, L, false, &launches, cfl, shared_tail);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (s != EU_OK) {
        if (g)
            cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess)
        return cuda_fail(h, e, "cudaStreamEndCapture");
    h->graph = g;
    CK(h, cudaGraphInstantiate(&h->graph_exec, g, 0));
    h->graph_launches = launches;
    h->graph_dirty = false;
    h->graph_cfl = cfl;
    h->graph_shared_tail = shared_tail;
    ++h->graph_gen;
    return EU_OK;
}

} // namespace

eu_status eu_chem_states(eu_handle *h, long long n, const double *T, const double *p, const double *Y, double *cs,
                         double *E)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!T || !p || !Y || !cs || !E || n < 0)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "null argument");
    if (!h->has_mech)
        return fail(h, EU_ERR_NOT_READY, "load a mechanism first");
    cudaSetDevice(h->cfg.device);
    LaunchArgs a = launch_args(h);
    CK(h, strict::launch_state_from_tpy(a, n, T, p, Y, cs, E));
    CK(h, cudaStreamSynchronize(h->stream));
    return EU_OK;
}

eu_status eu_chem_advance(eu_handle *h, long long n, double *cs, double *T, double *E, const double *dt, int *nchem)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!cs || !T || !E || !dt || n < 0)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "null argument");
    if (!h->has_mech)
        return fail(h, EU_ERR_NOT_READY, "load a mechanism first");
    cudaSetDevice(h->cfg.device);
    LaunchArgs a = launch_args(h);
    CK(h, cudaMemsetAsync(h->st.counters, 0, kCntCount * sizeof(unsigned long long), h->stream));
    CK(h, strict::launch_chem_samples(a, n, cs, T, E, dt, nchem));
    unsigned long long cnt[kCntCount];
    CK(h, cudaMemcpyAsync(cnt, h->st.counters, sizeof cnt, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    // With a per-sample nchem output the caller sees capped samples (nchem ==
    // max_substeps) and invalid ones (0) itself.
    if (cnt[kCntBadNchem] && !nchem)
        return fail(h, EU_ERR_NCHEM, "%llu samples predicted Nchem <= 0 or above max_substeps", cnt[kCntBadNchem]);
    return EU_OK;
}

eu_status eu_set_learned(eu_handle *h, eu_mlp *model, const eu_learned_config *lc)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!model || !lc || !lc->box_lo || !lc->box_hi || !lc->out_scale)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "null argument");
    if (!h->has_mech)
        return fail(h, EU_ERR_NOT_READY, "load a mechanism first");
    int n_in = 0, n_out = 0, members = 0;
    if (!mlp_shape(model, &n_in, &n_out, &members))
        return fail(h, EU_ERR_NOT_READY, "the model is not initialised");
    const int ns = h->mech.ns;
    if (n_in != ns + 3 || n_out != ns + 1)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "model must map %d inputs to %d outputs", ns + 3, ns + 1);
    cudaSetDevice(h->cfg.device);
    const long long cap = (long long)h->ni * h->nj * h->nk;
    LearnedParams &lp = h->lp;
    if (h->lp_capacity < cap || lp.members != members) {
        eu_status s;
        if ((s = dalloc(h, &lp.feat, size_t(cap) * (ns + 3))) != EU_OK) return s;
        if ((s = dalloc(h, &lp.pred, size_t(cap) * members * (ns + 1))) != EU_OK) return s;
        if ((s = dalloc(h, &lp.queue, size_t(cap))) != EU_OK) return s;
        if ((s = dalloc(h, &lp.fallback, size_t(cap))) != EU_OK) return s;
        if ((s = dalloc(h, &lp.active, size_t(cap))) != EU_OK) return s;
        if ((s = dalloc(h, &lp.counts, size_t(5))) != EU_OK) return s;
        h->lp_capacity = cap;
    }
    if (!h->h_counts)
        CK(h, cudaMallocHost(&h->h_counts, 2 * sizeof(int)));
    lp.members = members;
    lp.tau = lc->tau;
    lp.min_nchem = lc->min_nchem;
    lp.frozen_y = lc->frozen_y;
    lp.frozen_T = lc->frozen_T;
    lp.frozen_radical = lc->frozen_radical;
    for (int a = 0; a < ns + 3; ++a) {
        lp.box_lo[a] = lc->box_lo[a];
        lp.box_hi[a] = lc->box_hi[a];
    }
    for (int o = 0; o < ns + 1; ++o) {
        lp.out_scale[o] = lc->out_scale[o];
        lp.out_eps[o] = lc->out_eps ? lc->out_eps[o] : 0.0;
        lp.out_bound[o] = lc->out_bound ? lc->out_bound[o] : 0.0;
    }
    for (int s = 0; s < ns; ++s) {
        std::string up;
        if (s < (int)h->mech.species.size())
            for (char ch : h->mech.species[s]) up += char(std::toupper((unsigned char)ch));
        lp.radical[s] = (up == "H" || up == "O" || up == "OH" || up == "HO2" || up == "H2O2") ? 1 : 0;
    }
    element_projector(h->mech, lp.proj);
    for (int s = 0; s < ns; ++s) {
        bool used = false;
        for (int r = 0; r < h->mech.nr; ++r)
            used |= h->mech.stoi_f[s * h->mech.nr + r] != 0 || h->mech.stoi_b[s * h->mech.nr + r] != 0;
        lp.inert[s] = used ? 0 : 1;
    }
    h->model = model;
    h->graph_dirty = true; // the kernels take these settings by value
    // the model's weights were packed on its own stream
    CK(h, cudaStreamSynchronize(mlp_stream(model)));
    return EU_OK;
}

namespace {
// nsteps timesteps: with cfl == 0 of the fixed dt, else each of dt = cfl x the
// CFL minimum of its own starting state (the time advanced goes to *time).
eu_status step_impl(eu_handle *h, int nsteps, double dt, double cfl, eu_step_stats *stats, double *time,
                    const double *dt_src = nullptr);
} // namespace

eu_status eu_step(eu_handle *h, int nsteps, double dt, eu_step_stats *stats)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (nsteps < 0 || !(dt > 0))
        return fail(h, EU_ERR_INVALID_ARGUMENT, "nsteps must be >= 0 and dt > 0");
    return step_impl(h, nsteps, dt, 0.0, stats, nullptr);
}

eu_status eu_step_cfl(eu_handle *h, int nsteps, double cfl, eu_step_stats *stats, double *time_advanced)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (nsteps < 0 || !(cfl > 0) || !(cfl <= 10))
        return fail(h, EU_ERR_INVALID_ARGUMENT, "nsteps must be >= 0 and 0 < cfl <= 10");
    return step_impl(h, nsteps, 0.0, cfl, stats, time_advanced);
}

eu_status eu_step_dt_device(eu_handle *h, int nsteps, const double *device_dt, eu_step_stats *stats)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (nsteps < 0 || !device_dt)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "nsteps must be >= 0 and device_dt non-null");
    return step_impl(h, nsteps, 0.0, 0.0, stats, nullptr, device_dt);
}

eu_status eu_cfl_dt(eu_handle *h, double cfl, double *device_dt)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!device_dt || !(cfl > 0) || !(cfl <= 10))
        return fail(h, EU_ERR_INVALID_ARGUMENT, "device_dt must be non-null and 0 < cfl <= 10");
    if (!h->has_mech || !h->has_state)
        return fail(h, EU_ERR_NOT_READY, "mechanism and state must be set first");
    cudaSetDevice(h->cfg.device);
    const LaunchArgs a = launch_args(h);
    // the reduction leaves dt in the handle's slot; d_time is scratch here
    CK(h, strict::launch_cfl(a, cfl, h->d_cfl_slot, h->d_time));
    CK(h, cudaMemcpyAsync(device_dt, h->d_dt, sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    return EU_OK;
}

// ------------------------------------------------------------ halo exchange

eu_status eu_halo_bytes(const eu_handle *h, size_t *bytes)
{
    if (!h || !bytes)
        return EU_ERR_INVALID_ARGUMENT;
    if (!h->has_mech)
        return EU_ERR_NOT_READY;
    const size_t elem = h->st.prim32 ? sizeof(float) : sizeof(double);
    *bytes = size_t(7 + h->mech.ns) * h->bc * size_t(h->ny) * h->nz * elem;
    return EU_OK;
}

namespace {
eu_status halo_copy(eu_handle *h, int face, bool pack, void *buf)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!buf || (face != 0 && face != 1))
        return fail(h, EU_ERR_INVALID_ARGUMENT, "face must be 0 or 1 and the buffer non-null");
    if (!h->has_mech || !h->has_state)
        return fail(h, EU_ERR_NOT_READY, "mechanism and state must be set first");
    cudaSetDevice(h->cfg.device);
    CK(h, strict::launch_halo(launch_args(h), 7 + h->mech.ns, face, pack, buf));
    return EU_OK;
}
} // namespace

eu_status eu_halo_pack(eu_handle *h, int face, void *device_buf) { return halo_copy(h, face, true, device_buf); }
eu_status eu_halo_unpack(eu_handle *h, int face, const void *device_buf)
{
    return halo_copy(h, face, false, const_cast<void *>(device_buf));
}

namespace {
eu_status step_impl(eu_handle *h, int nsteps, double dt, double cfl, eu_step_stats *stats, double *time,
                    const double *dt_src)
{
    if (!h->has_mech || !h->has_state)
        return fail(h, EU_ERR_NOT_READY, "mechanism and state must be set before stepping");
    if (h->cfg.boundary == EU_BC_ODW && !h->g.exch_lo && !h->st.inflow)
        return fail(h, EU_ERR_NOT_READY, "the ODW ghost fill needs its inflow tables (eu_set_inflow)");
    cudaSetDevice(h->cfg.device);
    const bool prof = h->cfg.profile != 0 && stats != nullptr;
    const LaunchArgs a = launch_args(h);
    const bool react = h->cfg.chemistry == EU_CHEM_STIFF;
    const bool learned = h->cfg.chemistry == EU_CHEM_LEARNED;
    if (learned && !h->model)
        return fail(h, EU_ERR_NOT_READY, "learned chemistry needs eu_set_learned first");
    const Launchers &L = flavour(h);
    // A step is replayed from its captured graph unless the caller asked for
    // eager launches, times phases, or a learned model has no fused kernel
    // (then the step reads the queue length back on the host).
    const bool graphs = !h->cfg.eager && !prof && (!learned || mlp_has_fused(h->model));
    double phase[4] = {0, 0, 0, 0};
    int launches = 0;
    if (stats)
        CK(h, cudaEventRecord(h->ev0, h->stream));
    CK(h, cudaMemsetAsync(h->st.counters, 0, kCntCount * sizeof(unsigned long long), h->stream));
    if (cfl > 0) {
        CK(h, cudaMemsetAsync(h->d_time, 0, sizeof(double), h->stream));
    } else if (dt_src) {
        CK(h, cudaMemcpyAsync(h->d_dt, dt_src, sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    } else {
        CK(h, strict::launch_set_value(h->d_dt, dt, h->stream));
        ++launches;
    }
    if (h->st.prim32 && nsteps > 0)
        h->prim_stale = true;
    int n = 0;
    if (graphs && nsteps > 0 && (h->graph_dirty || !h->graph_exec || h->graph_cfl != cfl || h->graph_shared_tail)) {
        // the first step runs eagerly (one-time kernel attribute set-up), then
        // the step is captured
        eu_status s = step_launches(h, a, L, false, &launches, cfl);
        if (s != EU_OK)
            return s;
        n = 1;
        if ((s = capture_step(h, a, L, cfl)) != EU_OK)
            return s;
    }
    for (; n < nsteps; ++n) {
        if (graphs) {
            CK(h, cudaGraphLaunch(h->graph_exec, h->stream));
            launches += h->graph_launches;
            continue;
        }
        eu_status s = step_launches(h, a, L, prof, &launches, cfl);
        if (s != EU_OK)
            return s;
        if (prof) {
            CK(h, cudaEventSynchronize(h->pev[3]));
            for (int q = 0; q < 3; ++q) {
                float ms = 0;
                CK(h, cudaEventElapsedTime(&ms, h->pev[q], h->pev[q + 1]));
                phase[q] += ms;
            }
        }
    }
    if (time) {
        if (cfl > 0) {
            CK(h, cudaMemcpyAsync(time, h->d_time, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
            CK(h, cudaStreamSynchronize(h->stream));
        } else {
            *time = dt * nsteps;
        }
    }
    if (!stats)
        return EU_OK;
    CK(h, cudaEventRecord(h->ev1, h->stream));
    unsigned long long cnt[kCntCount];
    CK(h, cudaMemcpyAsync(cnt, h->st.counters, sizeof cnt, cudaMemcpyDeviceToHost, h->stream));
    int queued = 0, model_err = 0;
    if (learned && nsteps > 0) {
        CK(h, cudaMemcpyAsync(&queued, h->lp.counts + 3, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaMemcpyAsync(&model_err, mlp_error_flag(h->model), sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    }
    CK(h, cudaStreamSynchronize(h->stream));
    float ms = 0;
    CK(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    std::memset(stats, 0, sizeof *stats);
    stats->steps = nsteps;
    stats->max_nchem = int(cnt[kCntMaxNchem]);
    stats->sum_nchem = (long long)cnt[kCntSumNchem];
    stats->reacting = react ? (long long)h->ni * h->nj * h->nk : queued;
    stats->learned = (long long)cnt[kCntLearned];
    stats->fallback = (long long)cnt[kCntFallback];
    stats->routed = (long long)cnt[kCntRouted];
    stats->nonfinite = (long long)cnt[kCntNonfinite];
    stats->device_ms = ms;
    stats->launches = launches;
    for (int q = 0; q < 4; ++q) stats->phase_ms[q] = phase[q];
    if (model_err) {
        CK(h, cudaMemsetAsync(mlp_error_flag(h->model), 0, sizeof(int), h->stream));
        return fail(h, EU_ERR_TIMEOUT, "a tensor-core pipeline wait of the learned model gave up");
    }
    if (cnt[kCntNonfinite])
        return fail(h, EU_ERR_NONFINITE, "%llu cells with non-finite density or temperature", cnt[kCntNonfinite]);
    if (cnt[kCntBadNchem])
        return fail(h, EU_ERR_NCHEM, "%llu cells predicted Nchem <= 0 or above max_substeps", cnt[kCntBadNchem]);
    return EU_OK;
}
} // namespace

eu_status eu_get_field(eu_handle *h, const char *name, double *out)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!name || !out)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "null argument");
    if (!h->has_mech)
        return fail(h, EU_ERR_NOT_READY, "no state");
    cudaSetDevice(h->cfg.device);
    const long long n3 = h->n3;
    const int ns = h->mech.ns;
    const size_t b = size_t(n3) * sizeof(double);
    const std::string n(name);
    const char *prim_names[7] = {"P", "D", "U", "V", "W", "H", "Gamma"};
    if (h->prim_stale && n != "T" && n != "E" && n != "CS" && n != "Di" && n != "Mc" && n != "CMS" && n != "Nchem") {
        const LaunchArgs a = launch_args(h);
        CK(h, flavour(h).materialize(a));
        h->prim_stale = false;
    }
    for (int f = 0; f < 7; ++f)
        if (n == prim_names[f]) {
            CK(h, cudaMemcpyAsync(out, h->st.prim + f * n3, b, cudaMemcpyDeviceToHost, h->stream));
            CK(h, cudaStreamSynchronize(h->stream));
            return EU_OK;
        }
    const double *src = nullptr;
    size_t planes = 1;
    if (n == "T") src = h->st.T;
    else if (n == "E") src = h->st.E;
    else if (n == "Yi") { src = h->st.prim + 7 * n3; planes = ns; }
    else if (n == "CS") { src = h->st.cs; planes = ns + 4; }
    else if (n == "Di" || n == "Mc") { src = h->st.cs; planes = ns; }
    else if (n == "CMS") {
        if (!h->st.cms)
            return fail(h, EU_ERR_INVALID_ARGUMENT, "CMS needs record_sources in the config");
        src = h->st.cms;
        planes = ns;
    }
    if (src) {
        CK(h, cudaMemcpyAsync(out, src, planes * b, cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        if (n == "Mc") // Update_after_CS: Mc = Di / Mw * 1000 (src/Flowfield.cpp:1589)
            for (int s = 0; s < ns; ++s)
                for (long long c = 0; c < n3; ++c) out[s * n3 + c] = out[s * n3 + c] / h->mech.mw[s] * 1000;
        return EU_OK;
    }
    if (n == "Nchem") {
        std::vector<int> v(n3);
        CK(h, cudaMemcpyAsync(v.data(), h->st.nchem, n3 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        for (long long c = 0; c < n3; ++c) out[c] = v[c];
        return EU_OK;
    }
    const char *derived[5] = {"Wav", "Rgas", "Cp", "C", "Ma"};
    for (int w = 0; w < 5; ++w)
        if (n == derived[w]) {
            const LaunchArgs a = launch_args(h);
            CK(h, flavour(h).derived(a, w, h->d_scratch));
            CK(h, cudaMemcpyAsync(out, h->d_scratch, b, cudaMemcpyDeviceToHost, h->stream));
            CK(h, cudaStreamSynchronize(h->stream));
            return EU_OK;
        }
    return fail(h, EU_ERR_INVALID_ARGUMENT, "unknown field %s", name);
}

// ------------------------------------------------------------ state dumps
// The reference's EU3D_STATE_V1_LE dump (Euler::Output, src/Euler.cpp:1540-1598):
// a text header "EU3D_STATE_V1_LE", one line of sizes and times (17 significant
// digits), one line of column names, then one row of 22 + 5 ns little-endian
// doubles per interior node in (i, j, k) order, k fastest. Written as block
// block_x of a blocks_x x 1 x 1 decomposition (one rank per block).

namespace {
const char *kDumpMagic = "EU3D_STATE_V1_LE";
const char *kDumpFixed[17] = {"X", "Y", "Z", "D", "T", "U", "V", "W", "E", "Wav", "Rgas", "Cp", "P", "H", "Gamma",
                              "C", "Ma"};

std::string dump_columns(int ns)
{
    std::string line;
    for (int f = 0; f < 17; ++f) line += (f ? " " : "") + std::string(kDumpFixed[f]);
    for (const char *field : {"Di", "Yi", "Mc"})
        for (int n = 0; n < ns; ++n) line += " " + std::string(field) + std::to_string(n);
    for (int n = 0; n < ns + 4; ++n) line += " CS" + std::to_string(n);
    for (int n = 0; n < ns; ++n) line += " CMS" + std::to_string(n);
    return line + " Nchem";
}
} // namespace

eu_status eu_write_state(eu_handle *h, const char *path, int iteration, int num, double final_time, double dt)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!path)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "null path");
    if (!h->has_mech || !h->has_state)
        return fail(h, EU_ERR_NOT_READY, "no state");
    const int ns = h->mech.ns;
    const long long n3 = h->n3;
    // every column as haloed planes, in the dump's order
    std::vector<std::vector<double>> cols;
    auto field = [&](const char *name, int planes) -> eu_status {
        std::vector<double> v(size_t(planes) * n3);
        eu_status st = eu_get_field(h, name, v.data());
        if (st != EU_OK)
            return st;
        for (int p = 0; p < planes; ++p) cols.emplace_back(v.begin() + p * n3, v.begin() + (p + 1) * n3);
        return EU_OK;
    };
    const char *plane1[14] = {"D", "T", "U", "V", "W", "E", "Wav", "Rgas", "Cp", "P", "H", "Gamma", "C", "Ma"};
    for (const char *f : plane1) {
        eu_status st = field(f, 1);
        if (st != EU_OK)
            return st;
    }
    for (const char *f : {"Di", "Yi", "Mc"}) {
        eu_status st = field(f, ns);
        if (st != EU_OK)
            return st;
    }
    eu_status st = field("CS", ns + 4);
    if (st == EU_OK && h->st.cms)
        st = field("CMS", ns);
    else if (st == EU_OK) // no recorded sources: the reference's CMS array holds zeros until written
        for (int p = 0; p < ns; ++p) cols.emplace_back(size_t(n3), 0.0);
    if (st == EU_OK)
        st = field("Nchem", 1);
    if (st != EU_OK)
        return st;
    std::FILE *f = std::fopen(path, "wb");
    if (!f)
        return fail(h, EU_ERR_IO, "cannot open %s for writing", path);
    // header: NS, total_n*, local n*, block coordinates (x blocks only), blocks
    // per axis, rank (the x block) of ranks, iteration, output number, time, dt
    const int blocks_x = h->cfg.blocks_x > 1 ? h->cfg.blocks_x : 1;
    std::fprintf(f, "%s\n%d %d %d %d %d %d %d %d 0 0 %d 1 1 %d %d %d %d %.17g %.17g\n%s\n", kDumpMagic, ns,
                 h->cfg.total_ni, h->nj, h->nk, h->ni, h->nj, h->nk, h->cfg.block_x, blocks_x, h->cfg.block_x, blocks_x,
                 iteration, num, final_time, dt, dump_columns(ns).c_str());
    const int ncols = 22 + 5 * ns;
    std::vector<double> row(ncols);
    bool ok = true;
    for (int i = h->bc; i < h->bc + h->ni && ok; ++i)
        for (int j = h->bc; j < h->bc + h->nj && ok; ++j)
            for (int k = h->bc; k < h->bc + h->nk; ++k) {
                const long long c = (static_cast<long long>(i) * h->ny + j) * h->nz + k;
                row[0] = h->x[i];
                row[1] = h->y[j];
                row[2] = h->z[k];
                // D T U V W E Wav Rgas Cp P H Gamma C Ma
                for (int q = 0; q < 14; ++q) row[3 + q] = cols[q][c];
                for (int q = 14; q < (int)cols.size(); ++q) row[3 + q] = cols[q][c];
                if (std::fwrite(row.data(), sizeof(double), ncols, f) != size_t(ncols)) {
                    ok = false;
                    break;
                }
            }
    if (std::fclose(f) != 0 || !ok)
        return fail(h, EU_ERR_IO, "writing %s failed", path);
    return EU_OK;
}

eu_status eu_read_state(eu_handle *h, const char *path, int *iteration, int *num, double *final_time, double *dt)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!path)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "null path");
    if (!h->has_mech)
        return fail(h, EU_ERR_NOT_READY, "load a mechanism first");
    std::FILE *f = std::fopen(path, "rb");
    if (!f)
        return fail(h, EU_ERR_IO, "cannot open %s", path);
    char magic[64] = {0};
    int v[17];
    double t = 0, d = 0;
    const int ns = h->mech.ns;
    bool ok = std::fgets(magic, sizeof magic, f) && std::strncmp(magic, kDumpMagic, std::strlen(kDumpMagic)) == 0;
    ok = ok && std::fscanf(f, "%d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %lf %lf", &v[0], &v[1], &v[2],
                           &v[3], &v[4], &v[5], &v[6], &v[7], &v[8], &v[9], &v[10], &v[11], &v[12], &v[13], &v[14],
                           &v[15], &v[16], &t, &d) == 19;
    // rest of the sizes line, then the column line
    int ch = 0;
    while (ok && (ch = std::fgetc(f)) != '\n' && ch != EOF) {}
    std::string columns;
    while (ok && (ch = std::fgetc(f)) != '\n' && ch != EOF) columns += char(ch);
    if (!ok || ch == EOF) {
        std::fclose(f);
        return fail(h, EU_ERR_IO, "%s is not an EU3D_STATE_V1_LE dump", path);
    }
    if (v[0] != ns || v[4] != h->ni || v[5] != h->nj || v[6] != h->nk || columns != dump_columns(ns)) {
        std::fclose(f);
        return fail(h, EU_ERR_INVALID_ARGUMENT,
                    "%s holds ns %d and %d x %d x %d local nodes; the handle has ns %d and %d x %d x %d", path, v[0],
                    v[4], v[5], v[6], ns, h->ni, h->nj, h->nk);
    }
    const long long n3 = h->n3;
    const int ncols = 22 + 5 * ns;
    std::vector<double> row(ncols), P(n3, 0.0), D(n3, 0.0), U(n3, 0.0), V(n3, 0.0), W(n3, 0.0), H(n3, 0.0),
        G(n3, 0.0), T(n3, 0.0), E(n3, 0.0), Y(size_t(ns) * n3, 0.0), CS(size_t(ns + 4) * n3, 0.0);
    for (int i = h->bc; i < h->bc + h->ni && ok; ++i)
        for (int j = h->bc; j < h->bc + h->nj && ok; ++j)
            for (int k = h->bc; k < h->bc + h->nk; ++k) {
                if (std::fread(row.data(), sizeof(double), ncols, f) != size_t(ncols)) {
                    ok = false;
                    break;
                }
                const long long c = (static_cast<long long>(i) * h->ny + j) * h->nz + k;
                D[c] = row[3];
                T[c] = row[4];
                U[c] = row[5];
                V[c] = row[6];
                W[c] = row[7];
                E[c] = row[8];
                P[c] = row[12];
                H[c] = row[13];
                G[c] = row[14];
                for (int s = 0; s < ns; ++s) Y[s * n3 + c] = row[17 + ns + s];
                for (int q = 0; q < ns + 4; ++q) CS[q * n3 + c] = row[17 + 3 * ns + q];
            }
    std::fclose(f);
    if (!ok)
        return fail(h, EU_ERR_IO, "%s ends before its last node", path);
    eu_status st = eu_set_state(h, CS.data(), T.data(), E.data(), P.data(), D.data(), U.data(), V.data(), W.data(),
                                H.data(), G.data(), Y.data());
    if (st != EU_OK)
        return st;
    if (iteration) *iteration = v[15];
    if (num) *num = v[16];
    if (final_time) *final_time = t;
    if (dt) *dt = d;
    return EU_OK;
}

// ------------------------------------------------------ asynchronous output
// A snapshot of the fields an output file needs is copied, in stream order,
// into a device buffer of the handle (so the timestep may go on at once), then
// to pinned host memory on a second stream, and a host thread formats and
// writes the file once that copy has landed.

namespace {
// Tecplot output of Euler::Output (src/Euler.cpp:1600-1790): block data over
// every haloed node, i fastest, these variables after X, Y, Z
const char *kTecplotFields[6] = {"T", "D", "P", "U", "V", "Ma"};
constexpr int kTecplotSpecies = 7;
// EU3D_STATE_V1_LE dump: the 14 one-plane fields after X, Y, Z, in column order
const char *kDumpPlanes[14] = {"D", "T", "U", "V", "W", "E", "Wav", "Rgas", "Cp", "P", "H", "Gamma", "C", "Ma"};

// Snapshot layout: double planes of n3 values; for the state dump 14 planes,
// Di (ns), Yi (ns), CS (ns + 4), CMS (ns), then Nchem as n3 ints.
size_t snap_planes(int kind, int ns)
{
    return kind == EU_OUTPUT_TECPLOT ? 6 + kTecplotSpecies : 14 + 4 * size_t(ns) + 4 + 1; // + the Nchem ints
}

// One plane of field `name` into dst on the handle's stream (device to device).
eu_status snap_plane(eu_handle *h, const std::string &n, double *dst)
{
    const long long n3 = h->n3;
    const size_t b = size_t(n3) * sizeof(double);
    const char *prim_names[7] = {"P", "D", "U", "V", "W", "H", "Gamma"};
    for (int f = 0; f < 7; ++f)
        if (n == prim_names[f]) {
            CK(h, cudaMemcpyAsync(dst, h->st.prim + f * n3, b, cudaMemcpyDeviceToDevice, h->stream));
            return EU_OK;
        }
    if (n == "T" || n == "E") {
        CK(h, cudaMemcpyAsync(dst, n == "T" ? h->st.T : h->st.E, b, cudaMemcpyDeviceToDevice, h->stream));
        return EU_OK;
    }
    const char *derived[5] = {"Wav", "Rgas", "Cp", "C", "Ma"};
    for (int w = 0; w < 5; ++w)
        if (n == derived[w]) {
            const LaunchArgs a = launch_args(h);
            CK(h, flavour(h).derived(a, w, dst));
            return EU_OK;
        }
    return fail(h, EU_ERR_INVALID_ARGUMENT, "unknown field %s", n.c_str());
}

// The reference writes each value with an ostream's default format: six
// significant digits, %g style.
void put_g(std::string &out, double v)
{
    char buf[40];
    const int n = std::snprintf(buf, sizeof buf, "%g\n", v);
    out.append(buf, size_t(n));
}

eu_status write_tecplot_file(const char *path, const eu_handle *h, const double *snap, std::string &err)
{
    std::FILE *f = std::fopen(path, "wb");
    if (!f) {
        err = std::string("cannot open ") + path + " for writing";
        return EU_ERR_IO;
    }
    const long long n3 = h->n3;
    std::string out = "Variables = X,Y,Z,T,D,P,U,V,Ma,Y1,Y2,Y3,Y4,Y5,Y6,Y7\n";
    out += "ZONE I=" + std::to_string(h->nx) + "\tJ=" + std::to_string(h->ny) + "\tK=" + std::to_string(h->nz) +
           "\ndatapacking=block\n";
    bool ok = true;
    auto flush = [&]() {
        ok = ok && std::fwrite(out.data(), 1, out.size(), f) == out.size();
        out.clear();
    };
    // node (i, j, k) in the reference's loop order: k outermost, i fastest
    for (int v = 0; v < 3 + 6 + kTecplotSpecies && ok; ++v) {
        for (int k = 0; k < h->nz; ++k) {
            for (int j = 0; j < h->ny; ++j)
                for (int i = 0; i < h->nx; ++i) {
                    const long long c = (static_cast<long long>(i) * h->ny + j) * h->nz + k;
                    put_g(out, v == 0 ? h->x[i] : v == 1 ? h->y[j] : v == 2 ? h->z[k] : snap[(v - 3) * n3 + c]);
                }
            if (out.size() > (size_t(1) << 22))
                flush();
        }
    }
    flush();
    if (std::fclose(f) != 0 || !ok) {
        err = std::string("writing ") + path + " failed";
        return EU_ERR_IO;
    }
    return EU_OK;
}

eu_status write_dump_file(const char *path, const eu_handle *h, const double *snap, int iteration, int num,
                          double final_time, double dt, std::string &err)
{
    std::FILE *f = std::fopen(path, "wb");
    if (!f) {
        err = std::string("cannot open ") + path + " for writing";
        return EU_ERR_IO;
    }
    const int ns = h->mech.ns;
    const long long n3 = h->n3;
    const double *di = snap + 14 * n3, *yi = di + ns * n3, *cs = yi + ns * n3, *cms = cs + (ns + 4) * n3;
    const int *nchem = reinterpret_cast<const int *>(cms + ns * n3);
    const int blocks_x = h->cfg.blocks_x > 1 ? h->cfg.blocks_x : 1;
    std::fprintf(f, "%s\n%d %d %d %d %d %d %d %d 0 0 %d 1 1 %d %d %d %d %.17g %.17g\n%s\n", kDumpMagic, ns,
                 h->cfg.total_ni, h->nj, h->nk, h->ni, h->nj, h->nk, h->cfg.block_x, blocks_x, h->cfg.block_x, blocks_x,
                 iteration, num, final_time, dt, dump_columns(ns).c_str());
    const int ncols = 22 + 5 * ns;
    std::vector<double> row(ncols);
    bool ok = true;
    for (int i = h->bc; i < h->bc + h->ni && ok; ++i)
        for (int j = h->bc; j < h->bc + h->nj && ok; ++j)
            for (int k = h->bc; k < h->bc + h->nk; ++k) {
                const long long c = (static_cast<long long>(i) * h->ny + j) * h->nz + k;
                row[0] = h->x[i];
                row[1] = h->y[j];
                row[2] = h->z[k];
                for (int q = 0; q < 14; ++q) row[3 + q] = snap[q * n3 + c];
                int o = 17;
                for (int q = 0; q < ns; ++q) row[o++] = di[q * n3 + c];
                for (int q = 0; q < ns; ++q) row[o++] = yi[q * n3 + c];
                // Update_after_CS: Mc = Di / Mw * 1000 (src/Flowfield.cpp:1589)
                for (int q = 0; q < ns; ++q) row[o++] = di[q * n3 + c] / h->mech.mw[q] * 1000;
                for (int q = 0; q < ns + 4; ++q) row[o++] = cs[q * n3 + c];
                for (int q = 0; q < ns; ++q) row[o++] = cms[q * n3 + c];
                row[o] = nchem[c];
                if (std::fwrite(row.data(), sizeof(double), ncols, f) != size_t(ncols)) {
                    ok = false;
                    break;
                }
            }
    if (std::fclose(f) != 0 || !ok) {
        err = std::string("writing ") + path + " failed";
        return EU_ERR_IO;
    }
    return EU_OK;
}
} // namespace

eu_status eu_output_wait(eu_handle *h)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (h->out_thread.joinable())
        h->out_thread.join();
    const eu_status s = h->out_status;
    h->out_status = EU_OK;
    if (s != EU_OK)
        return fail(h, s, "%s", h->out_err.c_str());
    return EU_OK;
}

eu_status eu_output_async(eu_handle *h, int kind, const char *path, int iteration, int num, double final_time,
                          double dt)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (!path || (kind != EU_OUTPUT_STATE && kind != EU_OUTPUT_TECPLOT))
        return fail(h, EU_ERR_INVALID_ARGUMENT, "null path or unknown output kind %d", kind);
    if (!h->has_mech || !h->has_state)
        return fail(h, EU_ERR_NOT_READY, "no state");
    if (kind == EU_OUTPUT_TECPLOT && h->mech.ns < kTecplotSpecies)
        return fail(h, EU_ERR_UNSUPPORTED, "the Tecplot output writes 7 species; the mechanism has %d", h->mech.ns);
    // one output in flight per handle: the previous writer finishes first
    eu_status prev = eu_output_wait(h);
    if (prev != EU_OK)
        return prev;
    cudaSetDevice(h->cfg.device);
    const int ns = h->mech.ns;
    const long long n3 = h->n3;
    const size_t bytes = snap_planes(kind, ns) * size_t(n3) * sizeof(double);
    if (bytes > h->snap_bytes) {
        if (h->d_snap) cudaFree(h->d_snap);
        if (h->h_snap) cudaFreeHost(h->h_snap);
        h->d_snap = h->h_snap = nullptr;
        h->snap_bytes = 0;
        CK(h, cudaMalloc(&h->d_snap, bytes));
        CK(h, cudaMallocHost(&h->h_snap, bytes));
        h->snap_bytes = bytes;
    }
    if (!h->out_stream) {
        CK(h, cudaStreamCreateWithFlags(&h->out_stream, cudaStreamNonBlocking));
        CK(h, cudaEventCreateWithFlags(&h->ev_snap, cudaEventDisableTiming));
        CK(h, cudaEventCreateWithFlags(&h->ev_host, cudaEventDisableTiming));
    }
    if (h->prim_stale) {
        const LaunchArgs a = launch_args(h);
        CK(h, flavour(h).materialize(a));
        h->prim_stale = false;
    }
    const size_t b = size_t(n3) * sizeof(double);
    double *d = h->d_snap;
    eu_status st = EU_OK;
    if (kind == EU_OUTPUT_TECPLOT) {
        for (int q = 0; q < 6 && st == EU_OK; ++q) st = snap_plane(h, kTecplotFields[q], d + q * n3);
        if (st == EU_OK)
            CK(h, cudaMemcpyAsync(d + 6 * n3, h->st.prim + 7 * n3, kTecplotSpecies * b, cudaMemcpyDeviceToDevice,
                                  h->stream));
    } else {
        for (int q = 0; q < 14 && st == EU_OK; ++q) st = snap_plane(h, kDumpPlanes[q], d + q * n3);
        if (st == EU_OK) {
            double *di = d + 14 * n3, *yi = di + ns * n3, *cs = yi + ns * n3, *cms = cs + (ns + 4) * n3;
            CK(h, cudaMemcpyAsync(di, h->st.cs, ns * b, cudaMemcpyDeviceToDevice, h->stream));
            CK(h, cudaMemcpyAsync(yi, h->st.prim + 7 * n3, ns * b, cudaMemcpyDeviceToDevice, h->stream));
            CK(h, cudaMemcpyAsync(cs, h->st.cs, (ns + 4) * b, cudaMemcpyDeviceToDevice, h->stream));
            // no recorded sources: the reference's CMS array holds zeros until written
            if (h->st.cms)
                CK(h, cudaMemcpyAsync(cms, h->st.cms, ns * b, cudaMemcpyDeviceToDevice, h->stream));
            else
                CK(h, cudaMemsetAsync(cms, 0, ns * b, h->stream));
            CK(h, cudaMemcpyAsync(cms + ns * n3, h->st.nchem, size_t(n3) * sizeof(int), cudaMemcpyDeviceToDevice,
                                  h->stream));
        }
    }
    if (st != EU_OK)
        return st;
    CK(h, cudaEventRecord(h->ev_snap, h->stream));
    CK(h, cudaStreamWaitEvent(h->out_stream, h->ev_snap, 0));
    CK(h, cudaMemcpyAsync(h->h_snap, h->d_snap, bytes, cudaMemcpyDeviceToHost, h->out_stream));
    CK(h, cudaEventRecord(h->ev_host, h->out_stream));
    const std::string file(path);
    h->out_thread = std::thread([h, kind, file, iteration, num, final_time, dt]() {
        cudaSetDevice(h->cfg.device);
        const cudaError_t e = cudaEventSynchronize(h->ev_host);
        if (e != cudaSuccess) {
            h->out_status = EU_ERR_CUDA;
            h->out_err = std::string("output copy: ") + cudaGetErrorString(e);
            return;
        }
        h->out_status = kind == EU_OUTPUT_TECPLOT
                            ? write_tecplot_file(file.c_str(), h, h->h_snap, h->out_err)
                            : write_dump_file(file.c_str(), h, h->h_snap, iteration, num, final_time, dt, h->out_err);
    });
    return EU_OK;
}

eu_status eu_write_tecplot(eu_handle *h, const char *path)
{
    const eu_status s = eu_output_async(h, EU_OUTPUT_TECPLOT, path, 0, 0, 0.0, 0.0);
    if (s != EU_OK)
        return s;
    return eu_output_wait(h);
}

eu_status eu_sync(eu_handle *h)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->cfg.device);
    CK(h, cudaStreamSynchronize(h->stream));
    return EU_OK;
}

eu_status eu_device_info(const eu_handle *h, void **stream, size_t *device_bytes)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (stream) *stream = h->stream;
    if (device_bytes) *device_bytes = h->bytes;
    return EU_OK;
}

} // extern "C"

// ------------------------------------------------------------ instance batches
// Several handles on one device advanced together: one CUDA graph whose
// independent branches are the instances' captured timesteps, launched once
// per step on the batch's own stream, so the kernels of different instances
// overlap on the GPU. The kinetics of the cells the instances leave to the
// stiff integrator after their own recovery (the learned mode's fallback
// queue, the deferred cells of the warp-per-cell kinetics) form one shared
// stage after every branch: one fixed grid drains the fallback queues of all
// instances taken end to end, then one persistent grid their deferred cells,
// so the reacting cells of all instances spread over the whole GPU whatever
// instance they sit in. Each instance keeps its own buffers, queues and
// statistics.
struct eu_batch {
    // instances of one flavour, mechanism and substep cap share one launch
    // per kinetics stage; their table entries are contiguous
    struct Group {
        LaunchArgs a;           // the first member's (mechanism, flavour, stream replaced)
        const Launchers *L;
        int first = 0, count = 0;
        bool fallback = false;  // some member has a stiff-fallback queue
        bool heavy = false;     // some member defers cells
        int heavy_blocks = 0;
    };
    std::vector<eu_handle *> hs;
    std::vector<unsigned> gens;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> joins; // one per instance
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool shared = true;              // eu_batch_set_shared_kinetics
    std::vector<Group> groups;
    BatchCell *d_tab = nullptr;      // [instances] (members of the groups, in group order)
    int *d_next = nullptr;           // [2 per group]: fallback and deferred-cell positions taken
    int shared_launches = 0;         // kernels of the shared stage per step
    int launches = 0;                // kernels per step, the instances' and the shared stage's
    std::string err;
};

namespace {

eu_status bfail(eu_batch *b, eu_status s, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    b->err = buf;
    return s;
}

#define BCK(b, call)                                                                               \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return bfail((b), e_ == cudaErrorMemoryAllocation ? EU_ERR_OUT_OF_MEMORY : EU_ERR_CUDA, "%s: %s", #call, \
                         cudaGetErrorString(e_));                                                  \
    } while (0)

void drop_batch_graph(eu_batch *b)
{
    if (b->exec)
        cudaGraphExecDestroy(b->exec);
    if (b->graph)
        cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->groups.clear();
}

// Whether an instance leaves kinetics to the shared stage.
bool needs_shared_stage(const eu_handle *h)
{
    const bool learned = h->cfg.chemistry == EU_CHEM_LEARNED;
    return learned || (h->st.heavy && h->cfg.chemistry == EU_CHEM_STIFF);
}

// The shared kinetics stage: the groups' table on the device, then the
// stage's launches recorded into `out` (zeroing the positions taken first).
eu_status build_shared_stage(eu_batch *b, cudaGraph_t *out)
{
    *out = nullptr;
    std::vector<BatchCell> tab;
    std::vector<int> done(b->hs.size(), 0);
    for (size_t i = 0; i < b->hs.size(); ++i) {
        eu_handle *h = b->hs[i];
        if (done[i] || !needs_shared_stage(h))
            continue;
        eu_batch::Group grp;
        grp.a = launch_args(h);
        grp.L = &flavour(h);
        grp.first = int(tab.size());
        grp.heavy_blocks = h->heavy_blocks;
        for (size_t j = i; j < b->hs.size(); ++j) {
            eu_handle *o = b->hs[j];
            if (done[j] || !needs_shared_stage(o) || &flavour(o) != grp.L || o->spec != h->spec ||
                launch_args(o).max_substeps != grp.a.max_substeps ||
                std::memcmp(&o->dmech, &h->dmech, sizeof(DevMech)) != 0)
                continue;
            done[j] = 1;
            BatchCell c{};
            c.st = o->st;
            c.n3 = o->g.n3;
            c.dt = o->d_dt;
            if (o->cfg.chemistry == EU_CHEM_LEARNED) {
                c.queue = o->lp.fallback;
                c.count = o->lp.counts + 1;
                grp.fallback = true;
            }
            if (o->st.heavy)
                grp.heavy = true;
            else
                c.st.heavy = nullptr;
            tab.push_back(c);
        }
        grp.count = int(tab.size()) - grp.first;
        b->groups.push_back(grp);
    }
    b->shared_launches = 0;
    if (b->groups.empty())
        return EU_OK;
    if (b->d_tab)
        cudaFree(b->d_tab);
    if (b->d_next)
        cudaFree(b->d_next);
    b->d_tab = nullptr;
    b->d_next = nullptr;
    BCK(b, cudaMalloc(&b->d_tab, tab.size() * sizeof(BatchCell)));
    BCK(b, cudaMalloc(&b->d_next, b->groups.size() * 2 * sizeof(int)));
    BCK(b, cudaMemcpyAsync(b->d_tab, tab.data(), tab.size() * sizeof(BatchCell), cudaMemcpyHostToDevice, b->stream));
    BCK(b, cudaStreamSynchronize(b->stream));
    BCK(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaMemsetAsync(b->d_next, 0, b->groups.size() * 2 * sizeof(int), b->stream);
    for (size_t q = 0; q < b->groups.size() && e == cudaSuccess; ++q) {
        eu_batch::Group &grp = b->groups[q];
        grp.a.stream = b->stream;
        const BatchCell *t = b->d_tab + grp.first;
        int *next = b->d_next + 2 * q;
        if (grp.fallback && (e = grp.L->react_queue_batch(grp.a, t, grp.count, next, kCntFallback)) == cudaSuccess)
            ++b->shared_launches;
        if (e == cudaSuccess && grp.heavy &&
            (e = grp.L->react_heavy_batch(grp.a, t, grp.count, next, grp.heavy_blocks)) == cudaSuccess)
            ++b->shared_launches;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess || ee != cudaSuccess) {
        if (g)
            cudaGraphDestroy(g);
        const cudaError_t bad = e != cudaSuccess ? e : ee;
        cudaGetLastError();
        return bfail(b, EU_ERR_CUDA, "shared kinetics stage: %s", cudaGetErrorString(bad));
    }
    *out = g;
    return EU_OK;
}

} // namespace

extern "C" {

eu_status eu_batch_create(eu_handle *const *handles, int count, eu_batch **out)
{
    if (!handles || count < 1 || !out)
        return EU_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    for (int i = 0; i < count; ++i) {
        if (!handles[i] || handles[i]->cfg.device != handles[0]->cfg.device)
            return EU_ERR_INVALID_ARGUMENT;
        for (int j = 0; j < i; ++j)
            if (handles[j] == handles[i])
                return EU_ERR_INVALID_ARGUMENT;
    }
    eu_batch *b = new (std::nothrow) eu_batch;
    if (!b)
        return EU_ERR_OUT_OF_MEMORY;
    b->hs.assign(handles, handles + count);
    b->gens.assign(count, 0);
    b->device = handles[0]->cfg.device;
    b->joins.assign(count, nullptr);
    bool ok = cudaSetDevice(b->device) == cudaSuccess &&
              cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreate(&b->ev0) == cudaSuccess && cudaEventCreate(&b->ev1) == cudaSuccess;
    for (int i = 0; ok && i < count; ++i)
        ok = cudaEventCreateWithFlags(&b->joins[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        eu_batch_destroy(b);
        return EU_ERR_CUDA;
    }
    *out = b;
    return EU_OK;
}

eu_status eu_batch_destroy(eu_batch *b)
{
    if (!b)
        return EU_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    if (b->stream)
        cudaStreamSynchronize(b->stream);
    drop_batch_graph(b);
    if (b->d_tab) cudaFree(b->d_tab);
    if (b->d_next) cudaFree(b->d_next);
    for (cudaEvent_t e : b->joins)
        if (e) cudaEventDestroy(e);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return EU_OK;
}

const char *eu_batch_last_error(const eu_batch *b) { return b ? b->err.c_str() : kNoHandle; }

eu_status eu_batch_set_shared_kinetics(eu_batch *b, int on)
{
    if (!b)
        return EU_ERR_INVALID_ARGUMENT;
    if (b->shared != (on != 0)) {
        cudaSetDevice(b->device);
        cudaStreamSynchronize(b->stream);
        drop_batch_graph(b);
        b->shared = on != 0;
    }
    return EU_OK;
}

eu_status eu_batch_launches(const eu_batch *b, int *per_step, int *shared_stage)
{
    if (!b)
        return EU_ERR_INVALID_ARGUMENT;
    if (!b->exec)
        return EU_ERR_NOT_READY;
    if (per_step)
        *per_step = b->launches;
    if (shared_stage)
        *shared_stage = b->shared_launches;
    return EU_OK;
}

eu_status eu_batch_step(eu_batch *b, int nsteps, const double *dt, eu_step_stats *stats, double *device_ms)
{
    if (!b || !dt || nsteps < 0)
        return EU_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    const int n = int(b->hs.size());
    bool rebuild = !b->exec;
    for (int i = 0; i < n; ++i) {
        eu_handle *h = b->hs[i];
        if (!(dt[i] > 0))
            return bfail(b, EU_ERR_INVALID_ARGUMENT, "instance %d: dt must be > 0", i);
        if (!h->has_mech || !h->has_state)
            return bfail(b, EU_ERR_NOT_READY, "instance %d: mechanism and state must be set", i);
        if (h->cfg.chemistry == EU_CHEM_LEARNED && (!h->model || !mlp_has_fused(h->model)))
            return bfail(b, EU_ERR_UNSUPPORTED, "instance %d: learned chemistry needs a model with the fused kernel", i);
        const bool tail = b->shared && needs_shared_stage(h);
        if (h->graph_dirty || !h->graph_exec || h->graph_cfl != 0 || h->graph_shared_tail != tail) {
            const eu_status s = capture_step(h, launch_args(h), flavour(h), 0, tail);
            if (s != EU_OK)
                return bfail(b, s, "instance %d: %s", i, h->err.c_str());
        }
        rebuild |= b->gens[i] != h->graph_gen;
    }
    if (rebuild) {
        drop_batch_graph(b);
        BCK(b, cudaGraphCreate(&b->graph, 0));
        std::vector<cudaGraphNode_t> nodes(n);
        b->launches = 0;
        for (int i = 0; i < n; ++i) {
            BCK(b, cudaGraphAddChildGraphNode(&nodes[i], b->graph, nullptr, 0, b->hs[i]->graph));
            b->gens[i] = b->hs[i]->graph_gen;
            b->launches += b->hs[i]->graph_launches;
        }
        b->shared_launches = 0;
        if (b->shared) {
            cudaGraph_t stage = nullptr;
            const eu_status s = build_shared_stage(b, &stage);
            if (s != EU_OK)
                return s;
            if (stage) {
                cudaGraphNode_t node;
                const cudaError_t e = cudaGraphAddChildGraphNode(&node, b->graph, nodes.data(), nodes.size(), stage);
                cudaGraphDestroy(stage); // the node holds its own copy
                BCK(b, e);
                b->launches += b->shared_launches;
            }
        }
        BCK(b, cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    // order after each instance's earlier work, set its dt and call counters
    for (int i = 0; i < n; ++i) {
        eu_handle *h = b->hs[i];
        BCK(b, cudaEventRecord(b->joins[i], h->stream));
        BCK(b, cudaStreamWaitEvent(b->stream, b->joins[i], 0));
        BCK(b, cudaMemsetAsync(h->st.counters, 0, kCntCount * sizeof(unsigned long long), b->stream));
        BCK(b, strict::launch_set_value(h->d_dt, dt[i], b->stream));
        if (h->st.prim32 && nsteps > 0)
            h->prim_stale = true;
    }
    BCK(b, cudaEventRecord(b->ev0, b->stream));
    for (int q = 0; q < nsteps; ++q) BCK(b, cudaGraphLaunch(b->exec, b->stream));
    BCK(b, cudaEventRecord(b->ev1, b->stream));
    // later work on each instance's stream follows the batch
    for (int i = 0; i < n; ++i) BCK(b, cudaStreamWaitEvent(b->hs[i]->stream, b->ev1, 0));
    if (!stats && !device_ms)
        return EU_OK;
    std::vector<unsigned long long> cnt(size_t(n) * kCntCount);
    std::vector<int> queued(n, 0), model_err(n, 0);
    for (int i = 0; i < n; ++i) {
        eu_handle *h = b->hs[i];
        BCK(b, cudaMemcpyAsync(&cnt[size_t(i) * kCntCount], h->st.counters, kCntCount * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, b->stream));
        if (h->cfg.chemistry == EU_CHEM_LEARNED && nsteps > 0) {
            BCK(b, cudaMemcpyAsync(&queued[i], h->lp.counts + 3, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
            BCK(b, cudaMemcpyAsync(&model_err[i], mlp_error_flag(h->model), sizeof(int), cudaMemcpyDeviceToHost,
                                   b->stream));
        }
    }
    BCK(b, cudaStreamSynchronize(b->stream));
    float ms = 0;
    BCK(b, cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    if (device_ms)
        *device_ms = ms;
    eu_status worst = EU_OK;
    for (int i = 0; i < n; ++i) {
        eu_handle *h = b->hs[i];
        const unsigned long long *c = &cnt[size_t(i) * kCntCount];
        if (stats) {
            eu_step_stats &st = stats[i];
            std::memset(&st, 0, sizeof st);
            st.steps = nsteps;
            st.max_nchem = int(c[kCntMaxNchem]);
            st.sum_nchem = (long long)c[kCntSumNchem];
            st.reacting = h->cfg.chemistry == EU_CHEM_STIFF ? (long long)h->ni * h->nj * h->nk : queued[i];
            st.learned = (long long)c[kCntLearned];
            st.fallback = (long long)c[kCntFallback];
            st.routed = (long long)c[kCntRouted];
            st.nonfinite = (long long)c[kCntNonfinite];
            st.device_ms = ms;
            st.launches = nsteps * h->graph_launches;
        }
        eu_status s = EU_OK;
        if (model_err[i])
            s = fail(h, EU_ERR_TIMEOUT, "a tensor-core pipeline wait of the learned model gave up");
        else if (c[kCntNonfinite])
            s = fail(h, EU_ERR_NONFINITE, "%llu cells with non-finite density or temperature", c[kCntNonfinite]);
        else if (c[kCntBadNchem])
            s = fail(h, EU_ERR_NCHEM, "%llu cells predicted Nchem <= 0 or above max_substeps", c[kCntBadNchem]);
        if (s != EU_OK && worst == EU_OK) {
            worst = s;
            bfail(b, s, "instance %d: %s", i, h->err.c_str());
        }
    }
    return worst;
}

} // extern "C"

// ------------------------------------------------------------------ autotuner
// Launch shapes that change no arithmetic (every candidate gives bitwise the
// same state), timed on the handle's own state, which is restored afterwards:
// the x-march length of the flux kernels (the block count's fit to the SMs
// against each block's prologue of four planes) and the block size of the
// recovery kernels. Choices are kept per grid and mode for the process, so
// later handles of the same shape start from them.
extern "C" {

eu_status eu_autotune(eu_handle *h, int reps, eu_tune_report *report)
{
    if (!h)
        return EU_ERR_INVALID_ARGUMENT;
    if (reps < 1 || reps > 1000)
        return fail(h, EU_ERR_INVALID_ARGUMENT, "reps must be 1..1000");
    if (!h->has_mech || !h->has_state)
        return fail(h, EU_ERR_NOT_READY, "mechanism and state must be set before tuning");
    if (h->cfg.chemistry == EU_CHEM_LEARNED && !h->model)
        return fail(h, EU_ERR_NOT_READY, "learned chemistry needs eu_set_learned first");
    cudaSetDevice(h->cfg.device);
    CK(h, cudaStreamSynchronize(h->stream));
    const long long n3 = h->n3;
    const int ns = h->mech.ns;
    // snapshot of everything a flux or recovery launch writes
    struct Part { void *p; size_t bytes; };
    std::vector<Part> parts = {{h->st.cs, size_t(ns + 4) * n3 * 8}, {h->st.T, size_t(n3) * 8},
                               {h->st.E, size_t(n3) * 8}, {h->st.prim, size_t(7 + ns) * n3 * 8},
                               {h->st.nchem, size_t(n3) * 4}};
    if (h->st.prim32)
        parts.push_back({h->st.prim32, size_t(7 + ns) * n3 * 4});
    if (h->st.cms) // the stiff kinetics records its sources
        parts.push_back({h->st.cms, size_t(ns) * n3 * 8});
    if (h->st.zm_fresh) // whether the restored z ghosts match their interior
        parts.push_back({h->st.zm_fresh, sizeof(int)});
    size_t total = 0;
    for (const Part &q : parts) total += q.bytes;
    unsigned char *snap = nullptr;
    CK(h, cudaMalloc(&snap, total));
    size_t off = 0;
    cudaError_t e = cudaSuccess;
    for (const Part &q : parts) {
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(snap + off, q.p, q.bytes, cudaMemcpyDeviceToDevice, h->stream);
        off += q.bytes;
    }
    const int ci_cand[] = {8, 12, 16, 20, 24, 29, 32, 43, 64};
    const int rb_cand[] = {64, 96, 128};
    eu_tune_report rep;
    std::memset(&rep, 0, sizeof rep);
    LaunchArgs a = launch_args(h);
    const Launchers &L = flavour(h);
    const bool learned = h->cfg.chemistry == EU_CHEM_LEARNED;
    auto time_it = [&](auto &&launch, float *ms) -> cudaError_t {
        cudaError_t r = launch(); // warm-up
        if (r == cudaSuccess) r = cudaEventRecord(h->ev0, h->stream);
        for (int q = 0; q < reps && r == cudaSuccess; ++q) r = launch();
        if (r == cudaSuccess) r = cudaEventRecord(h->ev1, h->stream);
        if (r == cudaSuccess) r = cudaEventSynchronize(h->ev1);
        if (r == cudaSuccess) r = cudaEventElapsedTime(ms, h->ev0, h->ev1);
        *ms /= reps;
        return r;
    };
    int best_ci = 16, best_rb = 128;
    float best = 1e30f;
    for (int ci : ci_cand) {
        if (e != cudaSuccess || ci > h->ni + 15)
            continue;
        a.flux_ci = ci;
        float ms = 0;
        e = time_it([&] { return L.flux_update(a); }, &ms);
        if (rep.flux_candidates < 16) {
            rep.flux_ci[rep.flux_candidates] = ci;
            rep.flux_ms[rep.flux_candidates++] = ms;
        }
        if (ms < best) {
            best = ms;
            best_ci = ci;
        }
    }
    a.flux_ci = best_ci;
    // the flux launches moved the conserved state: back to the snapshot
    // before timing the recovery on it
    auto restore = [&] {
        size_t o = 0;
        for (const Part &q : parts) {
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(q.p, snap + o, q.bytes, cudaMemcpyDeviceToDevice, h->stream);
            o += q.bytes;
        }
    };
    restore();
    best = 1e30f;
    // register targets: the learned-mode classification (3..6 blocks per SM),
    // the stiff kinetics (2..4); recovery alone has one
    const bool stiff = h->cfg.chemistry == EU_CHEM_STIFF;
    int best_minb = stiff ? 2 : 4;
    const int minb_learned[] = {3, 4, 5, 6}, minb_stiff[] = {2, 3, 4}, minb_other[] = {4};
    const int *minbs = learned ? minb_learned : stiff ? minb_stiff : minb_other;
    const int n_minb = learned ? 4 : stiff ? 3 : 1;
    for (int rb : rb_cand)
        for (int mq = 0; mq < n_minb; ++mq) {
            if (e != cudaSuccess)
                break;
            a.recover_block = rb;
            a.recover_minb = minbs[mq];
            float ms = 0;
            e = time_it(
                [&] {
                    if (learned) {
                        cudaError_t r = cudaMemsetAsync(h->lp.counts, 0, 3 * sizeof(int), h->stream);
                        return r == cudaSuccess ? L.recover_classify(a, h->lp) : r;
                    }
                    if (stiff) { // the step's kernel: recovery and kinetics (deferred cells' queue emptied)
                        cudaError_t r = h->st.heavy ? cudaMemsetAsync(h->st.heavy, 0, 2 * sizeof(int), h->stream)
                                                    : cudaSuccess;
                        return r == cudaSuccess ? L.recover_react(a, true) : r;
                    }
                    return L.recover_react(a, false);
                },
                &ms);
            if (rep.recover_candidates < 16) {
                rep.recover_block[rep.recover_candidates] = rb;
                rep.recover_minblocks[rep.recover_candidates] = minbs[mq];
                rep.recover_ms[rep.recover_candidates++] = ms;
            }
            if (ms < best) {
                best = ms;
                best_rb = rb;
                best_minb = minbs[mq];
            }
        }
    restore();
    // the timed kinetics launches counted into the step statistics
    if (e == cudaSuccess)
        e = cudaMemsetAsync(h->st.counters, 0, kCntCount * sizeof(unsigned long long), h->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(h->stream);
    cudaFree(snap);
    if (e != cudaSuccess)
        return cuda_fail(h, e, "autotune");
    h->flux_ci = best_ci;
    h->recover_block = best_rb;
    h->recover_minb = best_minb;
    h->graph_dirty = true;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tuned[tune_key(h)] = {best_ci, best_rb, best_minb};
    }
    rep.chosen_flux_ci = best_ci;
    rep.chosen_recover_block = best_rb;
    rep.chosen_recover_minblocks = best_minb;
    if (report)
        *report = rep;
    return EU_OK;
}

} // extern "C"
