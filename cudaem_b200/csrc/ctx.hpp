// The context behind the opaque ms_ctx handle.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "engine.hpp"

struct ms_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    double last_ms = 0.0;
    int64_t last_launches = 0;
    std::string prop_key;                        // parameters of the cached propagator table
    bool propT_built = false;                    // the table's transposed copy is current too
    void* exptab = nullptr;                      // exp(2 pi i k / 1024), k < 1024
    int* d_err = nullptr;                        // device word: a bounded device-side wait ran out
    int inject = 0;                              // host-side fault injection (MS_INJECT_*), for tests

    struct Buf {
        void* p = nullptr;
        size_t bytes = 0;
    };
    std::map<std::string, Buf> bufs;             // device buffers reused across calls
    std::map<int, void*> twiddles;               // inter-level FFT twiddles per transform length
    std::map<std::string, msb::ElemTable> elem_cache;

    // STEM probe-batch graph: one batch's launch sequence (probe, slice loop, detector),
    // captured once and replayed for every batch whose launch arguments match `graph_key`
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        int64_t launches = 0;                    // kernels inside the captured graph
    };
    std::map<std::string, Graph> graphs;         // keyed by the launch arguments they bake in
    bool use_graphs = true;
    int pass_variant = 0;                        // msb::PassVariant of the slice-pass kernels (0: classic)
    bool pot_overlap = false;                    // potential chunks on a side stream beside the slice passes
    bool trans_store = true;                     // CBED/TEM/STEM slices as t = exp(iσV) (else as σV)
    int last_batch = 0;                          // probe batch used by the last STEM call
    std::vector<cudaStream_t> side;              // streams of the grid groups of an uneven batch
    cudaStream_t pot_stream = nullptr;           // potential chunks computed beside the slice passes
    std::vector<cudaEvent_t> chunk_ev;           // completion of each potential chunk
    std::map<std::string, int> batch_choice;     // autotuned probe batch per grid and slice count
    std::map<std::string, int> tile_choice;      // autotuned tile shape per grid and batch
    int tile_shape = -1;                         // forced msb::TileShape, or -1: autotuned
    int last_tile = 0;                           // tile shape of the last call's hot passes
    std::string tune_path;                       // JSON file that keeps the autotuner's choices ("": none)
    std::string device_tag;                      // device name and SM count, the prefix of every tuning key
    void drop_graph();

    // per-kernel event timing
    bool profile = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<std::pair<std::string, size_t>> ev_pending;  // kernel class, index of its start event
    std::map<std::string, std::pair<int64_t, double>> prof;   // launches, total ms
    cudaEvent_t prof_event();
    void prof_resolve();

    // A device buffer of at least `bytes`, kept for later calls.  Growing a buffer first
    // drains the stream so that no queued kernel still reads the old allocation.
    void* buf(const std::string& name, size_t bytes);
    void release_all();

    // Free device memory as cudaMemGetInfo reports it.  The reading is kept until this context
    // allocates or frees device memory: the query is a driver call that can wait behind other
    // processes' queries of the device (a monitoring tool polling clocks, for one), and every
    // simulation asks for it at its start, while the GPU is idle.
    size_t free_mem();
    void forget_free_mem() { free_known = false; }
    bool free_known = false;
    size_t free_seen = 0;
};

namespace msb {
void ctx_activate(ms_ctx* c);
// The autotuner's JSON cache (tune.cpp): device_tag names the device in every key; tune_load
// merges the file's entries for this device into the context, tune_save writes them back.
std::string device_tag(ms_ctx* c);
void tune_load(ms_ctx* c);
void tune_save(ms_ctx* c);
// A defocus series of HRTEM images: n offsets (Angstrom) added to the objective lens's C10.
struct DefocusSeries {
    int n = 0;
    const double* df = nullptr;
};
void sim_tem_like(ms_ctx* c, const ms_params& p, const ms_atoms& a, ms_output* out, bool force_cbed,
                  const DefocusSeries* series = nullptr);
void sim_stem(ms_ctx* c, const ms_params& p, const ms_atoms& a, ms_output* out);
void sim_thickness(ms_ctx* c, const ms_params& p, const ms_atoms& a, ms_output* out);
void sim_potential(ms_ctx* c, const ms_params& p, const ms_atoms& a, int conf, float* V, int64_t cap, int on_dev,
                   int* n_slices);
void sim_stem_forward_potential(ms_ctx* c, const ms_params& p, const float* V, int S, int on_dev, double z_init,
                                const double* xy, int np, float* I);
void sim_stem_backward(ms_ctx* c, const ms_params& p, const float* V, int S, int on_dev, double z_init,
                       const double* xy, int np, const float* target, double* loss, float* dV, double* dC10,
                       double* dC30);
void sim_many(ms_ctx* c, int n, const ms_params* ps, const ms_atoms* as, ms_output* outs, double* lat);
void stem_forward_noalloc(cudaStream_t st, const ms_params& p, const float* V, int S, double z_init, const double* xy,
                          int np, float* I);
size_t noalloc_scratch_bytes();
}  // namespace msb
