// extern "C" entry points of libcudaem_b200.so.  Every call is wrapped so that
// a C++ exception or a CUDA error becomes an ms_status plus a message kept in
// the context (ms_last_error); nothing is printed.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <exception>
#include <new>

#include "ctx.hpp"
#include "detmath.cuh"
#include "engine.hpp"

namespace {
thread_local std::string g_noctx_err;

template <class F>
ms_status guarded(ms_ctx* c, F&& f)
{
    // calls without a context keep their message per host thread (ms_last_error(NULL)); a success
    // clears it like a context's
    std::string& err = c ? c->err : g_noctx_err;
    try {
        f();
        err.clear();
        return MS_OK;
    } catch (const msb::MsError& e) {
        err = e.what();
        return e.st;
    } catch (const std::bad_alloc&) {
        err = "host allocation failed";
        return MS_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        err = e.what();
        return MS_ERR_INTERNAL;
    }
}
}  // namespace

extern "C" {

const char* ms_version(void) { return "cudaem_b200 1.0 (sm_100a)"; }
int ms_abi_version(void) { return MS_ABI_VERSION; }

void ms_default_params(ms_params* p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->simulation_type = MS_SIM_HRTEM;
    p->nx = p->ny = 512;
    p->lx = p->ly = 40.0;
    p->dz = 2.0;
    p->bwl = 1;
    p->E0 = 200.0;
    p->potential_type = MS_POT_MOLIERE;
    p->pot_rmin = 0.01;
    p->pot_rmax = 3.0;
    p->phonon_model = MS_PHONON_STILL;
    p->pn_nconf = 1;
    p->pn_seed = 42;
    p->pn_dim_x = p->pn_dim_y = p->pn_dim_z = 1;
    p->slice_border = -1;
    p->iw_type = -1;
    p->illumination_model = MS_ILLUM_COHERENT;
    p->temporal_spatial_incoh = MS_TSI_TEMPORAL_SPATIAL;
    p->obj_lens.dsf_npoints = p->cond_lens.dsf_npoints = 8;
    p->obj_lens.ssf_npoints = p->cond_lens.ssf_npoints = 4;
    p->data_record = MS_RECORD_INTENSITY;
    p->thick_det = 0;
    p->exec_mode = MS_EXEC_BATCHED;
    p->probe_batch = 0;
    p->ckpt_interval = 8;
    p->gpu_num = 1;
}

ms_status ms_validate_params(const ms_params* p)
{
    return guarded(nullptr, [&] {
        MS_REQUIRE(p != nullptr, MS_ERR_INVALID_ARG, "params is NULL");
        msb::validate_params(*p);
    });
}

ms_status ms_create(ms_ctx** out, int device)
{
    if (!out) return MS_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        g_noctx_err = "no CUDA device";
        return MS_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) return MS_ERR_NO_DEVICE;
    ms_ctx* c = new (std::nothrow) ms_ctx();
    if (!c) return MS_ERR_OUT_OF_MEMORY;
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return MS_ERR_CUDA;
    }
    c->stream = c->own_stream;
    *out = c;
    return MS_OK;
}

ms_status ms_destroy(ms_ctx* c)
{
    if (!c) return MS_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    c->release_all();
    for (auto e : c->ev_pool) cudaEventDestroy(e);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    for (auto s : c->side) cudaStreamDestroy(s);
    if (c->pot_stream) cudaStreamDestroy(c->pot_stream);
    for (auto e : c->chunk_ev) cudaEventDestroy(e);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return MS_OK;
}

const char* ms_last_error(const ms_ctx* c)
{
    if (!c) return g_noctx_err.c_str();
    return c->err.c_str();
}

ms_status ms_set_stream(ms_ctx* c, void* s)
{
    if (!c) return MS_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    c->stream = s ? (cudaStream_t)s : c->own_stream;
    return MS_OK;
}

ms_status ms_set_profiling(ms_ctx* c, int enable)
{
    if (!c) return MS_ERR_INVALID_ARG;
    c->profile = enable != 0;
    return MS_OK;
}

ms_status ms_profile_reset(ms_ctx* c)
{
    if (!c) return MS_ERR_INVALID_ARG;
    c->prof.clear();
    return MS_OK;
}

ms_status ms_profile_get(const ms_ctx* c, const char* kernel, int64_t* launches, double* total_ms)
{
    if (!c || !kernel) return MS_ERR_INVALID_ARG;
    auto it = c->prof.find(kernel);
    if (launches) *launches = it == c->prof.end() ? 0 : it->second.first;
    if (total_ms) *total_ms = it == c->prof.end() ? 0.0 : it->second.second;
    return MS_OK;
}

void* ms_get_stream(ms_ctx* c) { return c ? (void*)c->stream : nullptr; }
double ms_last_device_ms(const ms_ctx* c) { return c ? c->last_ms : 0.0; }
int64_t ms_last_launch_count(const ms_ctx* c) { return c ? c->last_launches : 0; }

int ms_last_probe_batch(const ms_ctx* c) { return c ? c->last_batch : 0; }

ms_status ms_set_pass_kernels(ms_ctx* c, int variant)
{
    if (!c || variant < 0 || variant > 3) return MS_ERR_INVALID_ARG;
    c->pass_variant = variant;
    if (c->stream) {
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->stream);
    }
    c->drop_graph();   // captured graphs hold the other kernels
    return MS_OK;
}

ms_status ms_set_transmission_store(ms_ctx* c, int enable)
{
    if (!c || enable < 0 || enable > 1) return MS_ERR_INVALID_ARG;
    c->trans_store = enable != 0;
    if (c->stream) {
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->stream);
    }
    c->drop_graph();
    return MS_OK;
}

ms_status ms_set_tile_shape(ms_ctx* c, int shape)
{
    if (!c || shape < -1 || shape > 7) return MS_ERR_INVALID_ARG;
    c->tile_shape = shape;
    if (c->stream) {
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->stream);
    }
    c->drop_graph();   // captured graphs hold the other kernels
    return MS_OK;
}

int ms_last_tile_shape(const ms_ctx* c) { return c ? c->last_tile : 0; }

ms_status ms_set_tune_cache(ms_ctx* c, const char* path)
{
    if (!c) return MS_ERR_INVALID_ARG;
    c->tune_path = path ? path : "";
    if (!c->tune_path.empty()) {
        cudaSetDevice(c->device);
        msb::tune_load(c);
    }
    return MS_OK;
}

ms_status ms_set_fault_injection(ms_ctx* c, int what)
{
    if (!c || what < MS_INJECT_NONE || what > MS_INJECT_ALLOC_FAIL) return MS_ERR_INVALID_ARG;
    c->inject = what;
    return MS_OK;
}

ms_status ms_set_potential_overlap(ms_ctx* c, int enable)
{
    if (!c) return MS_ERR_INVALID_ARG;
    c->pot_overlap = enable != 0;
    return MS_OK;
}

ms_status ms_set_graphs(ms_ctx* c, int enable)
{
    if (!c) return MS_ERR_INVALID_ARG;
    c->use_graphs = enable != 0;
    if (!c->use_graphs) {
        cudaSetDevice(c->device);
        if (c->stream) cudaStreamSynchronize(c->stream);
        c->drop_graph();
    }
    return MS_OK;
}

ms_status ms_physics(double E0_kV, double* lambda, double* sigma, double* gamma)
{
    if (!(E0_kV > 0)) return MS_ERR_INVALID_ARG;
    msb::Physics ph = msb::physics_of(E0_kV, 0.0);
    if (lambda) *lambda = ph.lambda;
    if (sigma) *sigma = ph.sigma;
    if (gamma) *gamma = ph.gamma;
    return MS_OK;
}

ms_status ms_simulate_tem(ms_ctx* c, const ms_params* p, const ms_atoms* a, ms_output* out)
{
    if (!c) return MS_ERR_INVALID_ARG;
    return guarded(c, [&] {
        MS_REQUIRE(p && a, MS_ERR_INVALID_ARG, "params or atoms is NULL");
        MS_REQUIRE(p->simulation_type == MS_SIM_HRTEM || p->simulation_type == MS_SIM_ED, MS_ERR_INVALID_ARG,
                   "ms_simulate_tem runs HRTEM or ED");
        msb::sim_tem_like(c, *p, *a, out, false);
    });
}

ms_status ms_simulate_tem_defocus_series(ms_ctx* c, const ms_params* p, const ms_atoms* a, int n_defocus,
                                         const double* defocus, ms_output* out)
{
    if (!c) return MS_ERR_INVALID_ARG;
    return guarded(c, [&] {
        MS_REQUIRE(p && a, MS_ERR_INVALID_ARG, "params or atoms is NULL");
        MS_REQUIRE(p->simulation_type == MS_SIM_HRTEM, MS_ERR_INVALID_ARG,
                   "ms_simulate_tem_defocus_series runs HRTEM");
        msb::DefocusSeries ser;
        ser.n = n_defocus;
        ser.df = defocus;
        msb::sim_tem_like(c, *p, *a, out, false, &ser);
    });
}

ms_status ms_simulate_cbed(ms_ctx* c, const ms_params* p, const ms_atoms* a, ms_output* out)
{
    if (!c) return MS_ERR_INVALID_ARG;
    return guarded(c, [&] {
        MS_REQUIRE(p && a, MS_ERR_INVALID_ARG, "params or atoms is NULL");
        MS_REQUIRE(p->simulation_type == MS_SIM_CBED, MS_ERR_INVALID_ARG, "ms_simulate_cbed runs CBED");
        msb::sim_tem_like(c, *p, *a, out, true);
    });
}

ms_status ms_simulate_stem(ms_ctx* c, const ms_params* p, const ms_atoms* a, ms_output* out)
{
    if (!c) return MS_ERR_INVALID_ARG;
    return guarded(c, [&] {
        MS_REQUIRE(p && a, MS_ERR_INVALID_ARG, "params or atoms is NULL");
        msb::sim_stem(c, *p, *a, out);
    });
}

ms_status ms_simulate_thickness(ms_ctx* c, const ms_params* p, const ms_atoms* a, ms_output* out)
{
    if (!c) return MS_ERR_INVALID_ARG;
    return guarded(c, [&] {
        MS_REQUIRE(p && a, MS_ERR_INVALID_ARG, "params or atoms is NULL");
        msb::sim_thickness(c, *p, *a, out);
    });
}

ms_status ms_displace_atoms(const ms_params* p, const ms_atoms* a, int conf, float* x, float* y, float* z)
{
    return guarded(nullptr, [&] {
        MS_REQUIRE(p && a && x && y && z, MS_ERR_INVALID_ARG, "NULL argument");
        MS_REQUIRE(conf >= 0, MS_ERR_INVALID_ARG, "conf must be >= 0");
        msb::validate_atoms(*p, a);
        msb::host_displace(*p, *a, conf, x, y, z);
    });
}

ms_status ms_build_slices(const ms_params* p, const ms_atoms* a, int conf, int* n_slices, float* bounds,
                          int bounds_capacity, int* atom_slice)
{
    return guarded(nullptr, [&] {
        MS_REQUIRE(p && a && n_slices, MS_ERR_INVALID_ARG, "NULL argument");
        MS_REQUIRE(p->dz > 0, MS_ERR_INVALID_ARG, "dz must be positive");
        msb::validate_atoms(*p, a);
        std::vector<float> x(a->n), y(a->n), z(a->n);
        msb::host_displace(*p, *a, conf, x.data(), y.data(), z.data());
        std::vector<float> b;
        int ns = msb::host_slices(*p, z.data(), a->n, &b, atom_slice);
        *n_slices = ns;
        if (bounds) {
            MS_REQUIRE(bounds_capacity >= (int)b.size(), MS_ERR_INVALID_ARG, "bounds capacity below n_slices+1");
            std::memcpy(bounds, b.data(), sizeof(float) * b.size());
        }
    });
}

ms_status ms_build_crystal(int n_basis, const int* basis_Z, const double* frac, double a, double b, double c,
                           int na, int nb, int nc, float sigma, float occ, int64_t* n_out, int* Z, float* x, float* y,
                           float* z, float* sig_out, float* occ_out)
{
    return guarded(nullptr, [&] {
        MS_REQUIRE(n_basis >= 1 && basis_Z && frac && n_out, MS_ERR_INVALID_ARG, "bad basis");
        MS_REQUIRE(na >= 1 && nb >= 1 && nc >= 1 && a > 0 && b > 0 && c > 0, MS_ERR_INVALID_ARG, "bad repeats");
        int64_t n = (int64_t)n_basis * na * nb * nc;
        *n_out = n;
        if (!x) return;
        MS_REQUIRE(Z && y && z && sig_out && occ_out, MS_ERR_INVALID_ARG, "NULL output array");
        int64_t k = 0;
        for (int iz = 0; iz < nc; iz++)
            for (int iy = 0; iy < nb; iy++)
                for (int ix = 0; ix < na; ix++)
                    for (int j = 0; j < n_basis; j++) {
                        Z[k] = basis_Z[j];
                        x[k] = (float)((ix + frac[3 * j]) * a);
                        y[k] = (float)((iy + frac[3 * j + 1]) * b);
                        z[k] = (float)((iz + frac[3 * j + 2]) * c);
                        sig_out[k] = sigma;
                        occ_out[k] = occ;
                        k++;
                    }
    });
}

ms_status ms_projected_potential(ms_ctx* c, const ms_params* p, const ms_atoms* a, int conf, float* V,
                                 int64_t capacity, int on_dev, int* n_slices)
{
    if (!c) return MS_ERR_INVALID_ARG;
    return guarded(c, [&] {
        MS_REQUIRE(p && a, MS_ERR_INVALID_ARG, "params or atoms is NULL");
        msb::sim_potential(c, *p, *a, conf, V, capacity, on_dev, n_slices);
    });
}

ms_status ms_stem_forward_potential(ms_ctx* c, const ms_params* p, const float* V, int n_slices, int on_dev,
                                    double z_init, const double* probe_xy, int n_probe, float* I)
{
    if (!c) return MS_ERR_INVALID_ARG;
    return guarded(c, [&] {
        MS_REQUIRE(p, MS_ERR_INVALID_ARG, "params is NULL");
        msb::sim_stem_forward_potential(c, *p, V, n_slices, on_dev, z_init, probe_xy, n_probe, I);
    });
}

ms_status ms_stem_forward_potential_noalloc(void* stream, const ms_params* p, const float* V, int n_slices,
                                            double z_init, const double* probe_xy, int n_probe, float* I)
{
    return guarded(nullptr, [&] {
        MS_REQUIRE(p, MS_ERR_INVALID_ARG, "params is NULL");
        msb::stem_forward_noalloc((cudaStream_t)stream, *p, V, n_slices, z_init, probe_xy, n_probe, I);
    });
}

ms_status ms_stem_backward(ms_ctx* c, const ms_params* p, const float* V, int n_slices, int on_dev, double z_init,
                           const double* probe_xy, int n_probe, const float* target, double* loss, float* dL_dV,
                           double* dL_dC10, double* dL_dC30)
{
    if (!c) return MS_ERR_INVALID_ARG;
    return guarded(c, [&] {
        MS_REQUIRE(p, MS_ERR_INVALID_ARG, "params is NULL");
        msb::sim_stem_backward(c, *p, V, n_slices, on_dev, z_init, probe_xy, n_probe, target, loss, dL_dV, dL_dC10,
                               dL_dC30);
    });
}

ms_status ms_simulate_many(ms_ctx* c, int n, const ms_params* params, const ms_atoms* atoms, ms_output* outs,
                           double* latency_ms)
{
    if (!c) return MS_ERR_INVALID_ARG;
    return guarded(c, [&] {
        MS_REQUIRE(n >= 1 && params && atoms && outs, MS_ERR_INVALID_ARG, "bad arguments");
        msb::sim_many(c, n, params, atoms, outs, latency_ms);
    });
}

}  // extern "C"
