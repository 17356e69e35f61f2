// engine.h -- one GRAPE-6 engine instance (one cluster_id) on one GPU.
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <vector>
#include "kernels.h"

namespace g6 {

struct EngineStats {
    long long calls = 0;
    long long interactions = 0;
    long long j_updates = 0;
    long long h2d_bytes = 0;
    long long d2h_bytes = 0;
    double last_force_ms = 0;
    double last_predict_ms = 0;
    double last_call_ms = 0;
    long long launches = 0;  // kernels launched by this instance
    // diagnostics (G6B200_TRACE=1 prints them when the instance closes)
    long long range_retries = 0, nb_calls = 0, predictions = 0, grows = 0;
    // calls of two i sharing one index: kira's binary perturbation call
    // (hdyn_grape6.C:3415-3587 sends both components with their top-level
    // node's index)
    long long pair_calls = 0;
    long long refined = 0;  // mixed mode: particles recomputed in FP64 (ill-conditioned sums)
    double wait_ms = 0, host_ms = 0;
};

class Engine {
  public:
    explicit Engine(int cluster_id);
    ~Engine();

    int open(int device, int nmax_hint);  // idempotent
    void close();
    int reset();
    bool is_open() const { return open_; }

    int set_npipes(int np);
    int npipes() const { return npipes_; }
    int set_mode(int mode);
    int mode() const { return mode_; }
    void set_ti(double ti) { ti_ = ti; }
    void set_default_h2(double h2) { default_h2_ = h2; }
    // Force a launch configuration (autotuner / experiments); il=0 clears.
    void set_config_override(const ForceConfig &c) { override_ = c; }

    int set_j(int address, int index, double tj, double mass, const double *k18,
              const double *j6, const double *a2, const double *v, const double *x);
    int flush_j();
    // Many j-particles at once (tj, mass [n]; k18, j6, a2, v, x [n][3] flat;
    // address/index/k18 may be null).  Same result as n set_j calls in
    // order: large uploads with distinct addresses go straight from the
    // caller's arrays to the device and one scatter kernel.
    int set_j_bulk(int n, const int *address, const int *index, const double *tj, const double *mass,
                   const double *k18, const double *j6, const double *a2, const double *v, const double *x);

    int firsthalf(int nj, int ni, const int *index, const double (*xi)[3],
                  const double (*vi)[3], double eps2, const double *h2);
    // GRAPE-4 pipeline (FP64 mode only): per-i softening eps2[i], pairs
    // with softened r2 == 0 skipped instead of an index exclusion, neighbour
    // test on the softened r2 (src/harpsims/harp3fastsim.c:240-300).  The
    // values are taken as the pipeline uses them (the GRAPE-4 ABI layer
    // applies that simulator's factor 2).  Results come from lasthalf.
    int firsthalf_g4(int nj, int ni, const double (*xi)[3], const double (*vi)[3], const double *eps2,
                     const double *h2);
    int lasthalf(int ni, double (*acc)[3], double (*jerk)[3], double *pot, int *nn);
    // Self-gravity sweep: forces on the j-addresses [i0, i0+ni) themselves,
    // predicted on the device (no host i-arrays).  Blocking.  With
    // copy_out false the results stay in device memory.
    int sweep(int nj, int i0, int ni, double eps2, bool copy_out, double (*acc)[3], double (*jerk)[3],
              double *pot, int *nn);
    // Potential only (no acc, jerk, nn): pot[ni] of the i-particles at the
    // j-memory predicted to the current ti.  Blocking.  ni <= npipes.
    int potential(int nj, int ni, const int *index, const double (*xi)[3], double eps2, double *pot);
    // Energies of the stored particles [0, nj) among themselves at the
    // current ti: epot = 1/2 sum m_i pot_i, ekin = 1/2 sum m_i |v_i|^2 (FP64,
    // fixed summation order), pot[nj] optionally copied out.  Blocking.
    int energies(int nj, double eps2, double *epot, double *ekin, double *pot);
    // Multi-GPU j-split of one cluster (split.cu; the caller runs the
    // collectives between the steps on `stream`, a cudaStream_t of this
    // device).  begin: force on the i-block from this instance's j-slice with
    // the slice cut into splits of block_j j (a multiple of 256), every
    // split's partial sums kept; writes agree[8 ni] (int64, device) and
    // returns when it is written.  fix: after the MAX all-reduce of agree,
    // sums[7 ni] and negj[ni] (int64, device) for the SUM / MAX all-reduces;
    // j_offset is the slice's first global address.  finish: the FP64
    // results from the reduced buffers, copied to host arrays (blocking).
    int split_begin(int nj, int ni, const int *index, const double (*xi)[3], const double (*vi)[3], double eps2,
                    int block_j, long long *agree, void *stream);
    int split_fix(long long nblocks_total, long long j_offset, const long long *agree, long long *sums,
                  long long *negj, void *stream);
    int split_finish(long long nblocks_total, long long nj_total, const long long *agree, const long long *sums,
                     const long long *negj, void *stream, double (*acc)[3], double (*jerk)[3], double *pot, int *nn);
    // Widen the mixed mode's fixed-point range to hold |x| <= xmax (ranks
    // of a split cluster pass the same value, so their grids agree).
    void set_position_range(double xmax);
    int read_neighbours();
    int get_neighbours(int pipe, int max_length, int *nblen, int *nbl);
    // Neighbour count of a pipe of the last call (after read_neighbours).
    int neighbour_count(int pipe) const;
    // The whole ascending list of a pipe of the last GRAPE-4 call, however
    // long (lists beyond the per-i capacity are recomputed for that pipe on
    // the device).  nbl has room for neighbour_count(pipe) entries.
    // Returns the count, or -1.
    int neighbours_all(int pipe, int *nbl);

    // For batched launches (server): flush staged j updates, widen the
    // fixed-point range for xi, predict j to the current ti if stale -- all
    // on this instance's stream, completion recorded in `ready` -- and fill
    // the j-side fields of `item` (jrec, nj, nj_pad, fs).  Returns 0.
    // With dst != nullptr the j-set is predicted into dst (nj_pad records of
    // this instance's kernel layout), always, and the cached prediction is
    // left alone -- so calls of one cluster at different block times can
    // share a launch.
    int prepare_batch_item(int nj, int ni, const double (*xi)[3], ForceParams &item, cudaEvent_t ready,
                           unsigned *status, void *dst = nullptr);
    // Runs the force kernel's bounded copy wait against a barrier that
    // nothing arrives at, through the same status word and wait path as a
    // call: returns 3 (the code of a timed-out copy wait) after limit_ms,
    // and leaves the instance ready for the next call.
    int selftest_copy_timeout(double limit_ms);
    // After a fixed-point range report: widen the range (x4) for the next call.
    void widen_range() {
        E_ += 2;
        pred_valid_ = false;
    }
    // Make this instance's stream wait for an event of another stream.
    int wait_event(cudaEvent_t e) { return cudaStreamWaitEvent(stream_, e, 0) == cudaSuccess ? 0 : -1; }
    bool identity_index() const { return n_nonident_ == 0; }
    int kernel_mode() const { return kmode(); }
    int device() const { return device_; }
    size_t footprint_bytes() const;

    const EngineStats &stats() const { return stats_; }
    const ForceConfig &last_config() const { return last_cfg_; }
    std::string last_error;

  private:
    int ensure_capacity(int address);
    int ensure_call_buffers(int ni, bool nb, size_t part_bytes);
    int firsthalf_impl(int nj, int ni, const int *index, const double (*xi)[3], const double (*vi)[3],
                       double eps2, const double *ieps2, const double *h2);
    int ensure_nb_buffers();
    int launch_call();  // predictor (if stale) + force + nb compaction + D2H
    int wait_call();    // wait; handle the fixed-point range retry
    int fail(const char *what, cudaError_t e);
    FixedScale scale() const;
    int choose_E(double xmax) const;

    int cluster_id_;
    bool open_ = false;
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    int num_sms_ = 148;
    int mode_ = kModeF64;
    int mixed_layout_ = kKernMixedP;  // record layout of the mixed mode
    int kmode() const { return mode_ == kModeF64 ? kKernF64 : mixed_layout_; }
    int npipes_ = 256;
    int nb_cap_ = 4096;
    double ti_ = 0;
    double default_h2_ = 0;
    ForceConfig override_{};

    // j-memory
    int cap_ = 0;
    double *d_jraw_ = nullptr;
    int *d_jindex_ = nullptr;
    void *d_jrec_ = nullptr;
    int n_nonident_ = 0;
    std::vector<char> nonident_;
    double xmax_ = 0;
    int E_ = -1000;

    // prediction cache
    bool pred_valid_ = false;
    double pred_ti_ = 0;
    int pred_nj_ = -1, pred_mode_ = -1, pred_E_ = 0;

    // j staging (pinned host -> device)
    int stage_cap_ = 0;
    int n_staged_ = 0;
    double *h_stage_vals_ = nullptr;
    int *h_stage_addr_ = nullptr, *h_stage_index_ = nullptr;
    double *d_stage_vals_ = nullptr;
    int *d_stage_addr_ = nullptr, *d_stage_index_ = nullptr;
    std::vector<int> slot_of_;
    cudaEvent_t ev_stage_ = nullptr;
    unsigned char *d_bulk_ = nullptr;  // device copies of a bulk upload's arrays
    size_t bulk_cap_ = 0;
    unsigned char *h_bulk_ = nullptr;  // pinned gather buffer of a bulk upload
    size_t h_bulk_cap_ = 0;
    bool bulk_busy_ = false;           // ev_stage_ marks the end of its last copy
    std::vector<unsigned> bulk_mark_;  // duplicate-address check (generation stamps)
    unsigned bulk_gen_ = 0;
    bool stage_busy_ = false;

    // per-call buffers
    int call_cap_ = 0;
    IRec *h_irec_ = nullptr, *d_irec_ = nullptr;
    double *h_ieps2_ = nullptr, *d_ieps2_ = nullptr;  // GRAPE-4 per-i softening
    unsigned char *h_out_ = nullptr, *d_out_ = nullptr;
    size_t part_cap_ = 0;
    Partial *d_part_ = nullptr;
    int *d_tile_cnt_ = nullptr;  // [call_cap_] i-tile arrival counters, kept at zero
    bool event_timing_ = false;  // per-call timing events (G6B200_EVENT_TIMING; sweeps always)
    bool timed_ = false;         // this call records timing events

    // neighbour lists
    int nb_alloc_ = 0;
    int *d_nb_count_ = nullptr, *d_nb_list_ = nullptr, *d_nb_sorted_ = nullptr;
    long long *d_nb_off_ = nullptr, *h_nb_off_ = nullptr;
    int *h_nb_count_ = nullptr;
    std::vector<int> nb_host_;
    bool nb_read_ = false;

    // call state
    bool pending_ = false;
    int call_ni_ = 0, call_nj_ = 0;
    double call_eps2_ = 0;
    bool call_nb_ = false;
    bool call_g4_ = false;
    // Small calls (<= kSmallMax i and staged j-updates): one launch carries
    // the host data as its parameter (G6B200_SMALL_CALLS=0 turns it off).
    bool small_enabled_ = true;
    bool refine_enabled_ = true;  // G6B200_REFINE=0: mixed mode without the FP64 recomputation
    long long mixed_min_work_ = 1LL << 25;  // mixed mode: calls of fewer interactions run in FP64
    bool call_f64_ = false;                 // this call runs on the FP64 records
    void mark_predicted(int nj, int km);
    int ensure_jrec64();
    bool call_small_ = false;
    int small_parity_ = 0;  // status word the next small call reports into
    int call_parity_ = 0;   // status word of the call in flight
    bool call_error_ = false;
    bool call_sweep_ = false;
    bool pot_request_ = false;  // the next firsthalf_impl call is a potential() call
    int split_request_ = 0;     // > 0: the next firsthalf_impl call is a split_begin() (block_j)
    int call_split_ = 0;        // block_j of the split call in flight (0: none)
    int split_nsplit_ = 0;      // splits of the last split call
    long long *split_agree_ = nullptr;  // caller's agree buffer of the split call
    cudaEvent_t ev_ext_ = nullptr;      // ordering against the caller's stream
    bool call_pot_ = false;     // potential-only kernel
    bool call_energy_ = false;  // + the energy reduction (sweeps)
    bool call_copy_ = true;
    double *d_energy_ = nullptr;  // [2 * kEnergyBlocks + 2] block partials, then epot, ekin
    // mixed-mode FP64 refinement (refine.cu)
    int ensure_refine_buffers(int ni);
    int ref_cap_ = 0;
    float *d_q_ = nullptr;            // [ref_cap_][2] error indicators
    int *d_ref_list_ = nullptr, *d_ref_tcnt_ = nullptr;
    IRec *d_ref_irec_ = nullptr;
    Partial *d_ref_part_ = nullptr;
    ForceParams *d_ref_items_ = nullptr;
    int *d_ref_small_ = nullptr;      // count, counter, pre[4] (pre[3]: the last call's flag count), done
    double *d_v2_ = nullptr;          // [kRefineBlocks + 1]
    void *d_jrec64_ = nullptr;        // FP64 records of the refinement [cap_]
    int jrec64_cap_ = 0;
    bool pred64_valid_ = false, v2_valid_ = false;
    double pred64_ti_ = 0;
    int pred64_nj_ = -1, v2_nj_ = -1;
    int *h_ref_count_ = nullptr;      // pinned
    bool call_refine_ = false;
    double *h_energy_ = nullptr;  // pinned: epot, ekin
    int call_i0_ = 0;
    ForceConfig last_cfg_{};
    cudaEvent_t ev_begin_ = nullptr, ev_pred0_ = nullptr, ev_pred1_ = nullptr;
    cudaEvent_t ev_force0_ = nullptr, ev_force1_ = nullptr, ev_done_ = nullptr;
    bool pred_timed_ = false;

    // host-side fault injection for the caller's retry paths (tests only)
    long long fault_lasthalf_at_ = -1, fault_pot_at_ = -1;
    long long lasthalf_count_ = 0;

    EngineStats stats_;
    SmallCall small_call_{};  // the parameter block of the last small call
};

}  // namespace g6
