// autotune.cu -- launch-shape autotuner.
//
// Tunes only choices that leave every result bit-identical:
//  * the row mapping and block size of the SpMVs that carry no reduction
//    (the BiCGSTAB SpMV): the canonical tile kernel or 1/2/4 rows per thread
//    in blocks of 128/256/512 threads;
//  * how a DILU application runs: one block sweeping every level (systems of
//    up to 262,144 rows), one launch per level, or every level in one
//    cooperative launch with a grid barrier between levels (systems of more
//    than 32,768 rows).
// Each candidate is timed with CUDA events on the case's own matrix at first
// use; choices are cached per size class (value size, log2 rows, entries per
// row), so later cases of the same class reuse them without timing.
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>

#include "case.hpp"
#include "kernels.hpp"

namespace xcal {

namespace {
using TuneKey = std::tuple<int, int, int, int>;  // (kind, value bytes, log2 n, entries per row)
std::mutex g_tune_mu;
std::map<TuneKey, SpmvShape> g_spmv_choice;
std::map<TuneKey, int> g_dilu_choice;

TuneKey key_of(int kind, int tsize, const Equation& E) {
    int l2 = E.n > 0 ? (int)std::floor(std::log2((double)E.n)) : 0;
    int epr = E.n > 0 ? (int)std::lround((double)E.nnz_csr / E.n) : 0;
    return TuneKey(kind, tsize, l2, epr);
}
}  // namespace

// average device time (ms) of f over reps launches, after one warm-up
template <class F>
static float time_ms(cudaStream_t s, cudaEvent_t a, cudaEvent_t b, int reps, F&& f) {
    f();
    XCAL_CUDA(cudaEventRecord(a, s));
    for (int i = 0; i < reps; ++i) f();
    XCAL_CUDA(cudaEventRecord(b, s));
    XCAL_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    XCAL_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms / reps;
}

template <class T>
static SpmvShape tune_spmv(Case& C, Equation& E, const T* nz, const T* x, T* y) {
    static const SpmvShape cands[] = {{0, 256}, {1, 128}, {1, 256}, {1, 512}, {2, 128},
                                      {2, 256}, {2, 512}, {4, 128}, {4, 256}, {4, 512}};
    const int reps = (int)std::max(3L, std::min(50L, 20000000L / std::max(E.nnz_csr, 1L)));
    CSRView A = E.view();
    SpmvShape best = cands[0];
    float best_ms = 1e30f;
    for (const SpmvShape& c : cands) {
        float ms = time_ms(C.stream, C.ev[6], C.ev[7], reps,
                           [&] { kr_spmv_shaped<T>(C.stream, c, A, nz, x, y, (const KScalars*)nullptr); });
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    return best;
}

// the fastest DILU form on this system: 1 one-block sweeps, 2 one launch per
// level, 3 one cooperative launch over every level
template <class T>
static int tune_dilu(Case& C, Equation& E, const T* nz, const T* D, const T* b, T* out) {
    const int reps = (int)std::max(3L, std::min(20L, 20000000L / std::max(E.nnz_csr, 1L)));
    const bool sb = E.use_block, sg = E.use_grid;
    int best = 2;
    float best_ms = 1e30f;
    for (int form = 1; form <= 3; ++form) {
        if (form == 1 && E.n > 4 * DILU_BLOCK_MAX_ROWS) continue;
        if (form == 3 && E.n <= DILU_BLOCK_MAX_ROWS / 2) continue;
        E.use_block = form == 1;
        E.use_grid = form == 3;
        float ms = time_ms(C.stream, C.ev[6], C.ev[7], reps, [&] { C.dilu_ldiv(E, nz, D, b, out, nullptr); });
        if (ms < best_ms) {
            best_ms = ms;
            best = form;
        }
    }
    E.use_block = sb;
    E.use_grid = sg;
    return best;
}

void Case::autotune() {
    if (tuned || capturing) return;
    tuned = true;
    // whether cooperative kernels run inside captured graphs: found here,
    // before any capture (the checks run graphs of their own)
    kr_coop_capture_ok(false);
    kr_coop_capture_ok(true);
    const bool mixed = cfg.precision == XCAL_PREC_MIXED;
    const int tsz = mixed ? 4 : 8;
    for (int e = 0; e < 2; ++e) {
        Equation& E = e == 0 ? U : P;
        const xcal_solver_setup& SS = e == 0 ? cfg.U_solver : cfg.p_solver;
        if (SS.solver == XCAL_SOLVER_BICGSTAB) {
            TuneKey k = key_of(0, tsz, E);
            std::unique_lock<std::mutex> lk(g_tune_mu);
            auto it = g_spmv_choice.find(k);
            if (it != g_spmv_choice.end()) {
                E.spmv_shape = it->second;
            } else {
                lk.unlock();
                SpmvShape sh = mixed ? tune_spmv<float>(*this, E, E.nz32.p, ws.fp.p, ws.fq.p)
                                     : tune_spmv<double>(*this, E, E.nz.p, ws.p.p, ws.q.p);
                E.spmv_shape = sh;
                lk.lock();
                g_spmv_choice[k] = sh;
            }
        }
        if (dilu_mode != 0) {
            E.use_block = dilu_mode == 1;
            E.use_grid = dilu_mode == 3;
        } else if (SS.precond == XCAL_PRECOND_DILU) {
            TuneKey k = key_of(1, tsz, E);
            std::unique_lock<std::mutex> lk(g_tune_mu);
            auto it = g_dilu_choice.find(k);
            int form;
            if (it != g_dilu_choice.end()) {
                form = it->second;
            } else {
                lk.unlock();
                form = mixed ? tune_dilu<float>(*this, E, E.nz32.p, E.P32.p, ws.fr.p, ws.fz.p)
                             : tune_dilu<double>(*this, E, E.nz.p, E.P.p, ws.r.p, ws.z.p);
                lk.lock();
                g_dilu_choice[k] = form;
            }
            E.use_block = form == 1;
            E.use_grid = form == 3;
        }
    }
    sync();
}

}  // namespace xcal
