// batch.cu -- continuous batching of independent steady cases (SIMPLE).
//
// The cases of a batch stay resident (fields, matrices, Krylov workspaces)
// and advance one SIMPLE iteration per call in lockstep.  The face-loop and
// correction kernels run per case, each case on its own stream (forked from
// and joined back into the batch stream with events, so the cases' small
// kernels overlap on the GPU); every Krylov solve
// (three momentum components, then pressure) is one batched solve over all
// cases: the same kernels' tile bodies driven through a per-system
// descriptor table and tile map (block-diagonal system, per-case offsets),
// with per-case Krylov scalars, so each case stops on its own test and its
// result is the one it gets when solved alone.  Cases enter (xcal_batch_add)
// and leave (xcal_batch_remove) between iterations; admission is bounded by a
// device-memory budget.
#include <algorithm>
#include <array>
#include <chrono>
#include <cstring>

#include "batch.hpp"
#include "case.hpp"
#include "dev_common.cuh"
#include "kernels.hpp"

namespace xcal {

struct Batch {
    xcal_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    int cap = 0;
    size_t budget = 0, used = 0;
    std::vector<Case*> cases;
    std::vector<size_t> footprint;   // bytes charged per case (case + mesh share)
    std::vector<cudaStream_t> own;   // each case's own stream (restored on removal)
    std::vector<cudaEvent_t> joined; // per case: its per-case phase is done
    cudaEvent_t forked = nullptr;    // the batch stream reached a per-case phase
    DBuf<KScalars> S;                // [cap] Krylov scalars, one block per case
    KScalars* hS = nullptr;          // pinned
    DBuf<double> res;                // [cap*4] scaled residuals of the iteration
    double* hres = nullptr;          // pinned
    // composition-dependent tables (rebuilt when cases enter or leave)
    bool dirty = true;
    int ntiles = 0;
    DBuf<int2> tmap;                 // all cases
    DBuf<int2> tmap_act;             // subset (mixed-precision outer steps)
    DBuf<unsigned char> sys[2][4];   // [fp64, fp32][Ux, Uy, Uz, p] descriptor tables
    DBuf<BAux> aux[4];               // [Ux, Uy, Uz, p] FP64-side tables
    DBuf<int2> dlo[2], dup[2];       // merged DILU levels per equation (large systems)
    std::vector<int> dlo_off[2], dup_off[2];
    DBuf<int> small_ids;             // systems that run DILU as one block
    int n_small = 0;
    int small_n = 0;                 // rows of the largest of them
    DBuf<unsigned int> bars;         // persistent CG: barrier state per system
    DBuf<int> mem_ids;               // persistent CG, cluster form: member systems grouped by cluster size
    int* hmem = nullptr;             // pinned staging of mem_ids
    // one stream per cluster-size group (1, 2, 4, 8, 16 blocks), so the
    // groups' launches run side by side
    cudaStream_t gstream[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t gjoined[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    DBuf<int> perr;                  // persistent CG: a barrier wait gave up
    std::vector<int2> h_tmap;
    long long iterations = 0;
    long diverged_total = 0;  // cases retired for a NaN/Inf residual
    double phase_ms[4] = {0, 0, 0, 0};  // host wall time: face loops, U solves, p solve, total
    // steady-state Krylov chunks replayed as CUDA graphs, per [precision][slot];
    // every pointer they use is fixed until the composition changes
    struct ChunkGraph {
        cudaGraphExec_t exec = nullptr;
        long long launches = 0;
    };
    ChunkGraph chunk_graph[2][4];
    // each case's face-loop phases (U assembly + first component, second and
    // third components, pressure assembly, correction), captured at first
    // use and replayed on the case's own stream: everything they read is
    // device state or fixed for the case, as in graph mode
    static constexpr int N_PHASES = 8;
    std::vector<std::array<ChunkGraph, N_PHASES>> case_graph;

    void drop_graphs() {
        for (auto& row : chunk_graph)
            for (auto& g : row)
                if (g.exec) {
                    cudaGraphExecDestroy(g.exec);
                    g.exec = nullptr;
                }
    }

    static void drop_case_graphs(std::array<ChunkGraph, N_PHASES>& gs) {
        for (auto& g : gs)
            if (g.exec) {
                cudaGraphExecDestroy(g.exec);
                g.exec = nullptr;
            }
    }

    template <class F>
    void replay(ChunkGraph& g, F&& body) {
        replay_on(g, stream, body);
    }

    // launch the graph captured from body() on stream s (capturing it first)
    template <class F>
    void replay_on(ChunkGraph& g, cudaStream_t s, F&& body) {
        if (!g.exec) {
            const long long t0 = t_launch_count;
            cudaGraph_t graph = nullptr;
            XCAL_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try {
                body();
            } catch (...) {
                cudaStreamEndCapture(s, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            XCAL_CUDA(cudaStreamEndCapture(s, &graph));
            const long long captured = t_launch_count - t0;
            g_launch_count.fetch_sub(captured, std::memory_order_relaxed);
            t_launch_count = t0;
            cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
            cudaGraphDestroy(graph);
            XCAL_CUDA(e);
            g.launches = captured;
        }
        XCAL_CUDA(cudaGraphLaunch(g.exec, s));
        g_launch_count.fetch_add(g.launches, std::memory_order_relaxed);
        t_launch_count += g.launches;
    }

    Batch(xcal_ctx* c, int capacity, size_t bytes) : ctx(c), cap(capacity), budget(bytes) {
        XCAL_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        XCAL_CUDA(cudaEventCreateWithFlags(&forked, cudaEventDisableTiming));
        S.alloc(cap);
        S.zero(stream);
        res.alloc(4 * (size_t)cap);
        res.zero(stream);
        XCAL_CUDA(cudaMallocHost(&hS, cap * sizeof(KScalars)));
        XCAL_CUDA(cudaMallocHost(&hres, 4 * cap * sizeof(double)));
        bars.alloc(2 * (size_t)cap);
        mem_ids.alloc(cap);
        XCAL_CUDA(cudaMallocHost(&hmem, cap * sizeof(int)));
        for (int g = 0; g < 5; ++g) {
            XCAL_CUDA(cudaStreamCreateWithFlags(&gstream[g], cudaStreamNonBlocking));
            XCAL_CUDA(cudaEventCreateWithFlags(&gjoined[g], cudaEventDisableTiming));
        }
        bars.zero(stream);
        perr.alloc(1);
        perr.zero(stream);
    }
    ~Batch() {
        if (stream) cudaStreamSynchronize(stream);
        drop_graphs();
        for (auto& gs : case_graph) drop_case_graphs(gs);
        for (size_t i = 0; i < cases.size(); ++i) cases[i]->stream = own[i];
        for (cudaEvent_t e : joined) cudaEventDestroy(e);
        if (forked) cudaEventDestroy(forked);
        if (hS) cudaFreeHost(hS);
        if (hmem) cudaFreeHost(hmem);
        for (int g = 0; g < 5; ++g) {
            if (gstream[g]) {
                cudaStreamSynchronize(gstream[g]);
                cudaStreamDestroy(gstream[g]);
            }
            if (gjoined[g]) cudaEventDestroy(gjoined[g]);
        }
        if (hres) cudaFreeHost(hres);
        if (stream) cudaStreamDestroy(stream);
    }
    void sync() { XCAL_CUDA(cudaStreamSynchronize(stream)); }

    // f(case) for every case, each on its own stream after the work queued on
    // the batch stream so far; the batch stream then waits for all of them.
    // The cases share no memory, so their kernels may run concurrently.
    // phase >= 0: f's launches are captured once per case and replayed.
    template <class F>
    void per_case(F&& f, int phase = -1) {
        XCAL_CUDA(cudaEventRecord(forked, stream));
        for (size_t i = 0; i < cases.size(); ++i) {
            Case* c = cases[i];
            XCAL_CUDA(cudaStreamWaitEvent(own[i], forked, 0));
            c->stream = own[i];
            try {
                if (phase < 0)
                    f(c);
                else
                    replay_on(case_graph[i][phase], own[i], [&] { f(c); });
            } catch (...) {
                c->stream = stream;
                throw;
            }
            c->stream = stream;
            XCAL_CUDA(cudaEventRecord(joined[i], own[i]));
        }
        for (size_t i = 0; i < cases.size(); ++i) XCAL_CUDA(cudaStreamWaitEvent(stream, joined[i], 0));
    }

    int index_of(const Case* c) const {
        for (size_t i = 0; i < cases.size(); ++i)
            if (cases[i] == c) return (int)i;
        return -1;
    }

    void check_compatible(const Case* c) const {
        if (c->cfg.algorithm != XCAL_ALGO_SIMPLE) fail(XCAL_ERR_UNSUPPORTED, "batch: steady SIMPLE cases only");
        if (cases.empty()) return;
        const xcal_config& a = cases[0]->cfg;
        const xcal_config& b = c->cfg;
        if (a.precision != b.precision || a.U_solver.solver != b.U_solver.solver ||
            a.U_solver.precond != b.U_solver.precond || a.p_solver.solver != b.p_solver.solver ||
            a.p_solver.precond != b.p_solver.precond || a.ncorrectors != b.ncorrectors)
            fail(XCAL_ERR_UNSUPPORTED,
                 "batch: cases must share precision, solvers, preconditioners and non-orthogonal correctors");
    }

    void add(Case* c, size_t charge) {
        if ((int)cases.size() >= cap) fail(XCAL_ERR_BUSY, "batch: no free slot");
        if (used + charge > budget) fail(XCAL_ERR_BUSY, "batch: device-memory budget exceeded");
        if (index_of(c) >= 0) fail(XCAL_ERR_INVALID, "batch: case already admitted");
        check_compatible(c);
        c->autotune();
        c->sync();
        if (c->graph_mode) c->set_graph_mode(false);
        cudaEvent_t ev = nullptr;
        XCAL_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        joined.push_back(ev);
        case_graph.emplace_back();
        own.push_back(c->stream);
        c->stream = stream;
        cases.push_back(c);
        footprint.push_back(charge);
        used += charge;
        dirty = true;
    }

    void remove(Case* c) {
        int i = index_of(c);
        if (i < 0) fail(XCAL_ERR_INVALID, "batch: case not admitted");
        sync();
        c->stream = own[i];
        used -= footprint[i];
        cudaEventDestroy(joined[i]);
        joined.erase(joined.begin() + i);
        drop_case_graphs(case_graph[i]);
        case_graph.erase(case_graph.begin() + i);
        cases.erase(cases.begin() + i);
        own.erase(own.begin() + i);
        footprint.erase(footprint.begin() + i);
        dirty = true;
    }

    // ---- composition tables ----------------------------------------------
    template <class T>
    void fill_sys(int prec, int slot) {
        const int nc = (int)cases.size();
        std::vector<BSys<T>> h(std::max(nc, 1));
        for (int i = 0; i < nc; ++i) {
            Case* c = cases[i];
            const bool isU = slot < 3;
            Equation& E = isU ? c->U : c->P;
            const xcal_solver_setup& SS = isU ? c->cfg.U_solver : c->cfg.p_solver;
            BSys<T>& B = h[i];
            std::memset(&B, 0, sizeof(B));
            B.A = E.view();
            B.n = E.n;
            B.ntiles = (E.n + RED_TILE - 1) / RED_TILE;
            B.S = S.p + i;
            B.part0 = c->ws.part0.p;
            B.part1 = c->ws.part1.p;
            if constexpr (sizeof(T) == 8) {
                B.nz = (const T*)E.nz.p;
                B.P = (const T*)E.P.p;
                T* v[KV_COUNT] = {(T*)c->ws.x.p, (T*)c->ws.r.p, (T*)c->ws.z.p, (T*)c->ws.p.p, (T*)c->ws.q.p,
                                  (T*)c->ws.v.p, (T*)c->ws.s.p, (T*)c->ws.t.p, nullptr, (T*)c->ws.q.p};
                for (int k = 0; k < KV_COUNT; ++k) B.vec[k] = v[k];
                B.vec[KV_C] = (T*)(isU ? c->U.b[slot].p : c->P.b[0].p);
            } else {
                B.nz = (const T*)E.nz32.p;
                B.P = (const T*)E.P32.p;
                T* v[KV_COUNT] = {(T*)c->ws.fx.p, (T*)c->ws.fr.p, (T*)c->ws.fz.p, (T*)c->ws.fp.p, (T*)c->ws.fq.p,
                                  (T*)c->ws.fv.p, (T*)c->ws.fs.p, (T*)c->ws.ft.p, (T*)c->ws.fd.p, (T*)c->ws.fd.p};
                for (int k = 0; k < KV_COUNT; ++k) B.vec[k] = v[k];
            }
            if (SS.solver == XCAL_SOLVER_CG && SS.precond == XCAL_PRECOND_NONE) B.vec[KV_Z] = B.vec[KV_R];
            B.lo = level_view<T>(E, 0);
            B.up = level_view<T>(E, 1);
        }
        sys[prec][slot].upload((const unsigned char*)h.data(), h.size() * sizeof(BSys<T>), stream);
    }

    void fill_aux(int slot) {
        const bool isU = slot < 3;
        const int comp = isU ? slot : 0;
        std::vector<BAux> h(cases.size());
        for (size_t i = 0; i < cases.size(); ++i) {
            Case* c = cases[i];
            Equation& E = isU ? c->U : c->P;
            const xcal_solver_setup& SS = isU ? c->cfg.U_solver : c->cfg.p_solver;
            const bool cg = SS.solver == XCAL_SOLVER_CG;
            BAux& B = h[i];
            std::memset(&B, 0, sizeof(BAux));
            B.A = E.view();
            B.nz = E.nz.p;
            B.nz32 = E.nz32.p;
            B.P = E.P.p;
            B.P32 = SS.precond != XCAL_PRECOND_NONE ? E.P32.p : nullptr;
            B.b = isU ? c->U.b[comp].p : c->P.b[0].p;
            B.field = isU ? c->Uc[comp].p : c->p.p;
            B.dx = c->ws.dx.p;
            B.x = c->ws.x.p;
            B.r0 = cg ? c->ws.r.p : c->ws.q.p;
            B.d32 = cg ? c->ws.fr.p : c->ws.fd.p;
            B.x32 = c->ws.fx.p;
            B.S = S.p + i;
            B.part0 = c->ws.part0.p;
            B.part1 = c->ws.part1.p;
            B.res_out = res.p + 4 * i + slot;
            if (SS.precond == XCAL_PRECOND_DILU && !E.lower_off.empty()) {
                B.lsrc = E.lsell.src.p;
                B.lcol = E.lsell.col.p;
                B.lslice = E.lsell.slice.p;
                B.lval = E.lsell.val.p;
                B.lval32 = E.lsell.val32.p;
                B.ldinv = E.lsell.dinv.p;
                B.ldinv32 = E.lsell.dinv32.p;
                B.usrc = E.usell.src.p;
                B.uslice = E.usell.slice.p;
                B.uval = E.usell.val.p;
                B.uval32 = E.usell.val32.p;
            }
            B.n = E.n;
            B.ntiles = (E.n + RED_TILE - 1) / RED_TILE;
        }
        if (h.empty()) h.resize(1);
        aux[slot].upload(h, stream);
    }

    void rebuild() {
        if (!dirty) return;
        drop_graphs();
        const int nc = (int)cases.size();
        h_tmap.clear();
        for (int i = 0; i < nc; ++i) {
            int nt = (cases[i]->U.n + RED_TILE - 1) / RED_TILE;
            for (int t = 0; t < nt; ++t) h_tmap.push_back(make_int2(i, t));
        }
        ntiles = (int)h_tmap.size();
        tmap.upload(h_tmap.empty() ? std::vector<int2>(1, make_int2(0, 0)) : h_tmap, stream);
        tmap_act.alloc(std::max(ntiles, 1));
        if (nc > 0) {
            const bool fp32 = cases[0]->cfg.precision == XCAL_PREC_MIXED;
            for (int slot = 0; slot < 4; ++slot) {
                if (fp32)
                    fill_sys<float>(1, slot);
                else
                    fill_sys<double>(0, slot);
                fill_aux(slot);
            }
            // small systems: one block per DILU application
            std::vector<int> ids;
            small_n = 0;
            for (int i = 0; i < nc; ++i)
                if (cases[i]->U.dilu_block()) {
                    ids.push_back(i);
                    small_n = std::max(small_n, cases[i]->U.n);
                }
            n_small = (int)ids.size();
            if (ids.empty()) ids.push_back(0);
            small_ids.upload(ids, stream);
            // DILU levels of the other systems merged across cases: level l
            // holds every such case's level-l rows
            for (int e = 0; e < 2; ++e) {
                for (int dir = 0; dir < 2; ++dir) {
                    size_t L = 0;
                    for (Case* c : cases) {
                        Equation& E = e == 0 ? c->U : c->P;
                        if (E.dilu_block()) continue;
                        const std::vector<int>& off = dir == 0 ? E.lower_off : E.upper_off;
                        if (off.size() > 1) L = std::max(L, off.size() - 1);
                    }
                    std::vector<int> moff(L + 1, 0);
                    std::vector<int2> rows;
                    for (size_t l = 0; l < L; ++l) {
                        for (int i = 0; i < nc; ++i) {
                            Equation& E = e == 0 ? cases[i]->U : cases[i]->P;
                            if (E.dilu_block()) continue;
                            const std::vector<int>& off = dir == 0 ? E.lower_off : E.upper_off;
                            const std::vector<int>& hr = dir == 0 ? E.h_lower_rows : E.h_upper_rows;
                            if (l + 1 >= off.size()) continue;
                            for (int k = off[l]; k < off[l + 1]; ++k) rows.push_back(make_int2(i, hr[k]));
                        }
                        moff[l + 1] = (int)rows.size();
                    }
                    if (rows.empty()) rows.push_back(make_int2(0, 0));
                    (dir == 0 ? dlo[e] : dup[e]).upload(rows, stream);
                    (dir == 0 ? dlo_off[e] : dup_off[e]) = moff;
                }
            }
        }
        sync();
        dirty = false;
    }

    // ---- batched Krylov solve --------------------------------------------
    template <class T>
    void apply_M(int prec, int slot, int e, int pt, const int2* tm, int nt, int in, int out, int use_S) {
        const BSys<T>* sy = (const BSys<T>*)sys[prec][slot].p;
        if (pt == XCAL_PRECOND_JACOBI)
            kb_jacobi_apply<T>(stream, sy, tm, nt, in, out, use_S);
        else if (pt == XCAL_PRECOND_DILU)
            kb_dilu<T>(stream, sy, small_ids.p, n_small, small_n, dlo[e].p, dlo_off[e], dup[e].p, dup_off[e], in, out,
                       use_S);
        else
            kb_copy<T>(stream, sy, tm, nt, in, out, use_S);
    }

    // start + host-polled iterations over the systems of tile map tm (the
    // single-case loop's chunking: 4 -> 32 CG, 1 -> 8 BiCGSTAB)
    template <class T>
    void krylov(int prec, int slot, const xcal_solver_setup& SS, const int2* tm, int nt,
                const std::vector<int>& members) {
        const int e = slot < 3 ? 0 : 1;
        const BSys<T>* sy = (const BSys<T>*)sys[prec][slot].p;
        const int pt = SS.precond;
        const bool cg = SS.solver == XCAL_SOLVER_CG;
        if (cg) {
            if (pt != XCAL_PRECOND_NONE) apply_M<T>(prec, slot, e, pt, tm, nt, KV_R, KV_Z, 0);
            kb_cg_start<T>(stream, sy, tm, nt);
        } else {
            apply_M<T>(prec, slot, e, pt, tm, nt, KV_R0, KV_R, 0);
            kb_bicg_start<T>(stream, sy, tm, nt);
        }
        int itmax = 0;
        for (int i : members) itmax = std::max(itmax, hS[i].itmax);
        // every member's whole CG loop in one cooperative launch (falls
        // through to the batched two-kernel loop when the tiles of all
        // members cannot be co-resident)
        if (cg && (pt == XCAL_PRECOND_JACOBI || pt == XCAL_PRECOND_NONE)) {
            bool all_persist = true;
            int width = 0;  // a block form the members ask for (tests), else the widest that fits
            for (int i : members) {
                all_persist = all_persist && cases[i]->persistent_cg != 0;
                if (cases[i]->persistent_cg > 1) width = cases[i]->persistent_cg;
            }
            const int jac = pt == XCAL_PRECOND_JACOBI ? 1 : 0;
            int max_tiles = 0;
            for (int i : members) max_tiles = std::max(max_tiles, (cases[i]->U.n + RED_TILE - 1) / RED_TILE);
            bool cluster = false;
            if (all_persist && (width == 0 || width == PERSIST_CLUSTER_ONLY) && max_tiles <= PERSIST_CLUSTER_MAX)
                cluster = cluster_cg<T>(sy, members, jac, itmax + 1);
            if (cluster) {
                XCAL_CUDA(cudaMemcpyAsync(hS, S.p, cases.size() * sizeof(KScalars), cudaMemcpyDeviceToHost,
                                          stream));
                sync();
                for (int i : members)
                    if (!hS[i].done) fail(XCAL_ERR_TIMEOUT, "batch: persistent CG did not report completion");
                return;
            }
            if (all_persist && width != PERSIST_CLUSTER_ONLY &&
                kb_cg_persist<T>(stream, sy, tm, nt, jac, bars.p, (int)cases.size(), perr.p, itmax + 1, width)) {
                int errflag = 0;
                XCAL_CUDA(cudaMemcpyAsync(hS, S.p, cases.size() * sizeof(KScalars), cudaMemcpyDeviceToHost,
                                          stream));
                XCAL_CUDA(cudaMemcpyAsync(&errflag, perr.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
                sync();
                if (errflag) fail(XCAL_ERR_TIMEOUT, "batch: persistent CG grid barrier wait gave up");
                for (int i : members)
                    if (!hS[i].done) fail(XCAL_ERR_TIMEOUT, "batch: persistent CG did not report completion");
                return;
            }
        }
        const int CHUNK = cg ? 32 : 8;
        int chunk = cg ? 4 : 1;
        long launched = 0;
        // iterations run over every system of the batch: systems outside
        // `members` are done and their blocks return at once, so a full chunk
        // is the same launch sequence for every solve of this slot (a cached
        // graph); the start kernels above used the members' tile map
        tm = tmap.p;
        nt = ntiles;
        for (;;) {
            if ((launched += chunk) > (long)itmax + 2 * CHUNK + 32)
                fail(XCAL_ERR_TIMEOUT, "batch: a Krylov solve did not report completion within itmax iterations");
            if (chunk == CHUNK) {
                replay(chunk_graph[prec][slot], [&] {
                    for (int c = 0; c < CHUNK; ++c) iterate<T>(prec, slot, SS, tm, nt);
                });
            } else {
                for (int c = 0; c < chunk; ++c) iterate<T>(prec, slot, SS, tm, nt);
            }
            XCAL_CUDA(cudaMemcpyAsync(hS, S.p, cases.size() * sizeof(KScalars), cudaMemcpyDeviceToHost, stream));
            sync();
            bool all = true;
            for (int i : members) all = all && hS[i].done;
            if (all) break;
            if (chunk < CHUNK) chunk *= 2;
        }
    }

    // every member's CG in the cluster form, members grouped by the cluster
    // size they need (1, 2, 4, 8 or 16 blocks: a cluster per member), one
    // launch per group, the groups on their own streams; false (nothing
    // launched) when the device cannot run some group's cluster size
    template <class T>
    bool cluster_cg(const BSys<T>* sy, const std::vector<int>& members, int jac, int max_iters) {
        std::vector<int> grp[5];
        for (int i : members) {
            const int t = (cases[i]->U.n + RED_TILE - 1) / RED_TILE;
            int g = 0;
            while ((1 << g) < t) ++g;
            grp[g].push_back(i);
        }
        for (int g = 0; g < 5; ++g)
            if (!grp[g].empty() && persist_cluster_size(kb_cg_persist_cluster_kernel<T>(), 1 << g) != (1 << g))
                return false;
        int off = 0;
        for (int g = 0; g < 5; ++g) {
            for (int i : grp[g]) hmem[off++] = i;
        }
        XCAL_CUDA(cudaMemcpyAsync(mem_ids.p, hmem, off * sizeof(int), cudaMemcpyHostToDevice, stream));
        XCAL_CUDA(cudaEventRecord(forked, stream));
        off = 0;
        for (int g = 0; g < 5; ++g) {
            if (grp[g].empty()) continue;
            XCAL_CUDA(cudaStreamWaitEvent(gstream[g], forked, 0));
            kb_cg_persist_cluster<T>(gstream[g], sy, mem_ids.p + off, (int)grp[g].size(), 1 << g, jac, max_iters);
            XCAL_CUDA(cudaEventRecord(gjoined[g], gstream[g]));
            XCAL_CUDA(cudaStreamWaitEvent(stream, gjoined[g], 0));
            off += (int)grp[g].size();
        }
        return true;
    }

    // one Krylov iteration of every system (early exit where done)
    template <class T>
    void iterate(int prec, int slot, const xcal_solver_setup& SS, const int2* tm, int nt) {
        const int e = slot < 3 ? 0 : 1;
        const BSys<T>* sy = (const BSys<T>*)sys[prec][slot].p;
        const int pt = SS.precond;
        const bool cg = SS.solver == XCAL_SOLVER_CG;
        {
            {
                if (cg) {
                    kb_cg_spmv<T>(stream, sy, tm, nt);
                    if (pt == XCAL_PRECOND_JACOBI) {
                        kb_cg_update<T>(stream, sy, tm, nt, 1);
                    } else {
                        kb_cg_update<T>(stream, sy, tm, nt, 0);
                        if (pt == XCAL_PRECOND_DILU) apply_M<T>(prec, slot, e, pt, tm, nt, KV_R, KV_Z, 1);
                        kb_cg_rz<T>(stream, sy, tm, nt);
                    }
                } else {
                    kb_spmv<T>(stream, sy, tm, nt, KV_P, KV_Q);
                    apply_M<T>(prec, slot, e, pt, tm, nt, KV_Q, KV_V, 1);
                    kb_bicg_alpha<T>(stream, sy, tm, nt);
                    kb_bicg_s<T>(stream, sy, tm, nt);
                    kb_spmv<T>(stream, sy, tm, nt, KV_S, KV_Q);
                    apply_M<T>(prec, slot, e, pt, tm, nt, KV_Q, KV_T, 1);
                    kb_bicg_omega<T>(stream, sy, tm, nt);
                    kb_bicg_xr<T>(stream, sy, tm, nt);
                    kb_bicg_p<T>(stream, sy, tm, nt);
                }
            }
        }
    }

    // solve_system! for slot (0..2: U component, 3: p) of every case
    void solve(int slot) {
        const int nc = (int)cases.size();
        const bool isU = slot < 3;
        const int comp = isU ? slot : 0;
        const bool mixed = cases[0]->cfg.precision == XCAL_PREC_MIXED;
        const xcal_solver_setup& SS0 = isU ? cases[0]->cfg.U_solver : cases[0]->cfg.p_solver;
        std::vector<int> all(nc);
        for (int i = 0; i < nc; ++i) {
            all[i] = i;
            Case* c = cases[i];
            c->smooth(isU ? XCAL_EQN_U : XCAL_EQN_P, comp);
            const xcal_solver_setup& SS = isU ? c->cfg.U_solver : c->cfg.p_solver;
            std::memset(&hS[i], 0, sizeof(KScalars));
            hS[i].atol = SS.atol;
            hS[i].rtol = SS.rtol;
            hS[i].itmax = SS.itmax == 0 ? 2 * (isU ? c->U.n : c->P.n) : SS.itmax;
            if (mixed) {
                hS[i].mixed = 1;
                hS[i].inner_rtol = c->cfg.inner_rtol > 0 ? c->cfg.inner_rtol : 1e-3;
            }
        }
        if (!mixed) {
            XCAL_CUDA(cudaMemcpyAsync(S.p, hS, nc * sizeof(KScalars), cudaMemcpyHostToDevice, stream));
            if (SS0.precond == XCAL_PRECOND_DILU) kb_level_refresh(stream, aux[slot].p, tmap.p, ntiles, 0);
            kb_init_resid(stream, aux[slot].p, tmap.p, ntiles);
            krylov<double>(0, slot, SS0, tmap.p, ntiles, all);
            kb_finish(stream, aux[slot].p, tmap.p, ntiles);
            for (int i = 0; i < nc; ++i) cases[i]->last_iters[slot] = hS[i].iter;
        } else {
            kb_to_float(stream, aux[slot].p, tmap.p, ntiles);
            if (SS0.precond == XCAL_PRECOND_DILU) kb_level_refresh(stream, aux[slot].p, tmap.p, ntiles, 1);
            std::vector<char> active(nc, 1);
            std::vector<int> total(nc, 0);
            for (int outer = 0; outer < 64; ++outer) {
                std::vector<int> mem;
                for (int i = 0; i < nc; ++i)
                    if (active[i]) mem.push_back(i);
                if (mem.empty()) break;
                for (int i : mem) {
                    hS[i].outer = outer;
                    hS[i].iter = 0;
                    hS[i].done = 0;
                    hS[i].status = KS_RUNNING;
                }
                XCAL_CUDA(cudaMemcpyAsync(S.p, hS, nc * sizeof(KScalars), cudaMemcpyHostToDevice, stream));
                std::vector<int2> ta;
                for (const int2& t : h_tmap)
                    if (active[t.x]) ta.push_back(t);
                XCAL_CUDA(cudaMemcpyAsync(tmap_act.p, ta.data(), ta.size() * sizeof(int2), cudaMemcpyHostToDevice,
                                          stream));
                kb_defect(stream, aux[slot].p, tmap_act.p, (int)ta.size());
                krylov<float>(1, slot, SS0, tmap_act.p, (int)ta.size(), mem);
                // field += e for every member whose defect was not already at
                // its target (the device reads the same outer_conv flag)
                kb_correct(stream, aux[slot].p, tmap_act.p, (int)ta.size());
                for (int i : mem) {
                    if (hS[i].outer_conv) {
                        active[i] = 0;
                        continue;
                    }
                    total[i] += hS[i].iter;
                    int st = hS[i].status;
                    if (st == KS_ZERO_CURV || st == KS_BREAKDOWN || st == KS_TIRED ||
                        (st == KS_SOLVED && hS[i].eps <= hS[i].eps_outer))
                        active[i] = 0;
                }
            }
            for (int i = 0; i < nc; ++i) cases[i]->last_iters[slot] = total[i];
        }
        // residual (Solve_1_api.jl:441-464), FP64
        kb_residual(stream, aux[slot].p, tmap.p, ntiles);
    }

    // one SIMPLE iteration of every case (Solvers_1_SIMPLE.jl:164-240)
    void simple_iteration(double* res_out, int* conv_out) {
        if (cases.empty()) return;
        using clk = std::chrono::steady_clock;
        auto ms = [](clk::time_point a, clk::time_point b) {
            return std::chrono::duration<double, std::milli>(b - a).count();
        };
        const clk::time_point t0 = clk::now();
        rebuild();
        bool fresh = false;
        for (Case* c : cases) {
            fresh = fresh || !c->initialised;
            c->iteration += 1;
        }
        if (fresh)
            per_case([&](Case* c) {
                if (!c->initialised) c->initial_calculations();
            });
        double fv = 0, us = 0;
        for (int d = 0; d < 3; ++d) {
            clk::time_point a = clk::now();
            per_case(
                [&](Case* c) {
                    if (d == 0) c->discretise(XCAL_EQN_U);
                    c->bc_relax_U(d);
                    if (d == 0) c->update_precond(XCAL_EQN_U);
                },
                d);
            clk::time_point b = clk::now();
            solve(d);
            fv += ms(a, b);
            us += ms(b, clk::now());
        }
        const clk::time_point t1 = clk::now();
        per_case(
            [&](Case* c) {
                c->pressure_predictor(true);
                c->flux_divergence();
                XCAL_CUDA(cudaMemcpyAsync(c->prev.p, c->p.p, c->mesh->nC * sizeof(double), cudaMemcpyDeviceToDevice,
                                          c->stream));
                c->discretise(XCAL_EQN_P);
                c->apply_bcs(XCAL_EQN_P, 0);
                c->set_reference();
                c->update_precond(XCAL_EQN_P);
            },
            3);
        const clk::time_point t2 = clk::now();
        solve(3);
        const int ncorr = cases[0]->cfg.ncorrectors;
        if (ncorr > 0) {
            // non-orthogonal correctors (Solvers_1_SIMPLE.jl:196-206): every
            // corrector's pressure solve is one batched solve
            auto relax_grad = [&](Case* c) {
                c->explicit_relaxation_p(c->cfg.p_solver.relax);
                c->grad_p();
            };
            per_case(relax_grad, 5);
            for (int k = 0; k < ncorr; ++k) {
                per_case(
                    [&](Case* c) {
                        c->discretise(XCAL_EQN_P);
                        c->apply_bcs(XCAL_EQN_P, 0);
                        c->nonorth_correct();
                    },
                    6);
                solve(3);
                per_case(relax_grad, 5);
            }
        }
        const clk::time_point t3 = clk::now();
        per_case(
            [&](Case* c) {
                if (ncorr == 0) {
                    c->explicit_relaxation_p(c->cfg.p_solver.relax);
                    c->grad_p();
                }
                c->correct();
                if (!c->has_k()) c->turbulence();
            },
            ncorr > 0 ? 7 : 4);
        // turbulence with transported k (and omega): each case's own k /
        // omega solves (host-polled Krylov on its stream, on the p system's
        // storage, which the next iteration's pressure assembly rewrites),
        // so this phase runs uncaptured
        bool any_k = false;
        for (Case* c : cases) any_k = any_k || c->has_k();
        if (any_k)
            per_case([&](Case* c) {
                if (c->has_k()) c->turbulence();
            });
        XCAL_CUDA(cudaMemcpyAsync(hres, res.p, 4 * cases.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
        sync();
        const clk::time_point t4 = clk::now();
        ++iterations;
        phase_ms[1] += us;
        phase_ms[2] += ms(t2, t3);
        phase_ms[3] += ms(t0, t4);
        phase_ms[0] = phase_ms[3] - phase_ms[1] - phase_ms[2];
        (void)fv;
        (void)t1;
        // A case whose residual is NaN/Inf leaves the batch now, reported as
        // XCAL_ERR_DIVERGED in its row; the others are not touched (every
        // batched kernel keeps each case's data and scalars apart), so they
        // carry on exactly as they would have without it.
        std::vector<Case*> diverged;
        for (size_t i = 0; i < cases.size(); ++i) {
            Case* c = cases[i];
            const double* r = hres + 4 * i;
            bool bad = false;
            for (int k = 0; k < 4; ++k) {
                if (res_out) res_out[4 * i + k] = r[k];
                bad |= std::isnan(r[k]) || std::isinf(r[k]);
            }
            // Uz enters the test on 3D meshes only (Solvers_1_SIMPLE.jl:220-223)
            const bool uz = c->mesh->dim == 2 || r[2] <= c->cfg.U_solver.convergence;
            bool conv = r[0] <= c->cfg.U_solver.convergence && r[1] <= c->cfg.U_solver.convergence && uz &&
                        r[3] <= c->cfg.p_solver.convergence && c->cfg.turbulence == XCAL_TURB_LAMINAR;
            if (conv_out) conv_out[i] = bad ? XCAL_ERR_DIVERGED : (conv ? 1 : 0);
            if (bad) diverged.push_back(c);
        }
        for (Case* c : diverged) remove(c);
        diverged_total += (long)diverged.size();
    }
};

// Device bytes a case will hold, from the mesh sizes (upper bound of the
// allocations of upload_mesh and Case::Case; SELL padding bounded by 2%).
size_t estimate_case_bytes(long nC, long nF, long nB, int mixed, int dilu_U, int dilu_p) {
    const long nI = nF - nB;
    const double nnz = (double)(nC + 2 * nI) * 1.02 + 64.0;
    double b = 0;
    // mesh
    b += 88.0 * nF + 9.0 * 2 * nI + 16.0 * (nC + 1) + 8.0 * nC + 12.0 * nB;
    // equations U and p: slots (col 4, value 8, transpose 4 [+ fp32 value 4]),
    // rows (len 1, diag 4, diag0 8, P 8 [+ P32 4], b 8 per component, slices),
    // slot maps (cf_slot 2 nI, fslot nI), DILU level lists (8 per row)
    for (int e = 0; e < 2; ++e) {
        int nvec = e == 0 ? 3 : 1;
        b += nnz * (16.0 + (mixed ? 4.0 : 0.0));
        b += nC * (21.0 + 8.0 * nvec + (mixed ? 4.0 : 0.0)) + 4.0 * (nC / 32 + 2);
        b += 4.0 * 3 * nI;
        if ((e == 0 && dilu_U) || (e == 1 && dilu_p)) {
            // level lists and offsets, and the level-ordered triangles: per
            // off-diagonal slot column, source slot, value [+ fp32 value]
            b += 8.0 * nC + 16.0 * nC;
            // (SELL padding of the level order: up to half again), and 1/D
            // per lower slot [+ fp32]
            b += (nnz - nC) * 1.5 * (16.0 + (mixed ? 4.0 : 0.0)) + 2.0 * nC + 8.0 * (nC / 32 + 2);
            b += (nnz - nC) * 0.5 * 1.5 * (8.0 + (mixed ? 4.0 : 0.0));
            // the factor's transposed-entry slots (lower triangle) and
            // diagonal slots per position
            b += (nnz - nC) * 0.5 * 1.5 * 4.0 + 4.0 * nC;
        }
    }
    // three boundary-condition tables (85 bytes per boundary face) + partner lists
    b += 3.0 * (85.0 * nB + 4.0 * (nC + 1));
    // fields: 26 doubles per cell, 8 per face; Krylov: 9 doubles per cell
    // [+ 9 floats and two (r, p) float pairs, folded-CG partials]; tile
    // partials and small buffers
    b += nC * (26.0 + 9.0) * 8.0 + nF * 8.0 * 8.0 + (mixed ? 52.0 * nC + 16384.0 : 0.0);
    b += 3.0 * 8.0 * (nC / 2048 + 1) + 4096.0;
    // permutations (mesh) and the field staging buffer (case)
    b += 8.0 * nC + 8.0 * nF + 8.0 * std::max(nC, nF);
    return (size_t)b;
}

}  // namespace xcal

struct xcal_batch {
    std::unique_ptr<xcal::Batch> b;
};

using namespace xcal;

#define XCAL_BGUARD(ctx, ...)                                                 \
    try {                                                                     \
        __VA_ARGS__;                                                          \
        return XCAL_OK;                                                       \
    } catch (const ::xcal::Error& e) {                                        \
        if (ctx) ctx->set_error(e.msg);                                       \
        return e.code;                                                        \
    } catch (const std::exception& e) {                                       \
        if (ctx) ctx->set_error(e.what());                                    \
        return XCAL_ERR_INVALID;                                              \
    }

extern "C" {

int32_t xcal_footprint_estimate(int64_t n_cells, int64_t n_faces, int64_t n_bfaces, int32_t precision,
                                int32_t dilu_U, int32_t dilu_p, int64_t* bytes) {
    if (!bytes || n_cells <= 0 || n_faces < n_bfaces || n_bfaces < 0) return XCAL_ERR_INVALID;
    *bytes = (int64_t)estimate_case_bytes(n_cells, n_faces, n_bfaces, precision == XCAL_PREC_MIXED ? 1 : 0,
                                          dilu_U, dilu_p);
    return XCAL_OK;
}

int32_t xcal_case_footprint(const xcal_case* cs, int64_t* case_bytes, int64_t* mesh_bytes) {
    if (!cs) return XCAL_ERR_INVALID;
    if (case_bytes) *case_bytes = (int64_t)cs->c->bytes;
    if (mesh_bytes) *mesh_bytes = (int64_t)cs->c->mesh->bytes;
    return XCAL_OK;
}

int32_t xcal_batch_create(xcal_ctx* ctx, int32_t max_cases, int64_t budget_bytes, xcal_batch** out) {
    if (!ctx || !out || max_cases <= 0 || budget_bytes <= 0) return XCAL_ERR_INVALID;
    *out = nullptr;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return XCAL_ERR_CUDA;
    XCAL_BGUARD(ctx, {
        std::unique_ptr<Batch> b(new Batch(ctx, max_cases, (size_t)budget_bytes));
        xcal_batch* h = new xcal_batch();
        h->b = std::move(b);
        *out = h;
    })
}

int32_t xcal_batch_destroy(xcal_batch* b) {
    delete b;
    return XCAL_OK;
}

int32_t xcal_batch_add(xcal_batch* bt, xcal_case* cs, int64_t charge_bytes) {
    if (!bt || !cs) return XCAL_ERR_INVALID;
    Batch* b = bt->b.get();
    XCAL_BGUARD(b->ctx, {
        size_t charge = charge_bytes > 0 ? (size_t)charge_bytes : cs->c->bytes + cs->c->mesh->bytes;
        b->add(cs->c.get(), charge);
        // the batch's FP32 inner solves use the canonical kernels; the case
        // keeps that form if it later runs alone, so its arithmetic never
        // depends on whether it was batched
        cs->c->set_inner_cg(1);
    })
}

int32_t xcal_batch_remove(xcal_batch* bt, xcal_case* cs) {
    if (!bt || !cs) return XCAL_ERR_INVALID;
    Batch* b = bt->b.get();
    XCAL_BGUARD(b->ctx, { b->remove(cs->c.get()); })
}

int32_t xcal_batch_info(const xcal_batch* bt, int32_t* n_cases, int64_t* used_bytes, int64_t* budget_bytes) {
    if (!bt) return XCAL_ERR_INVALID;
    if (n_cases) *n_cases = (int32_t)bt->b->cases.size();
    if (used_bytes) *used_bytes = (int64_t)bt->b->used;
    if (budget_bytes) *budget_bytes = (int64_t)bt->b->budget;
    return XCAL_OK;
}

int32_t xcal_batch_timings(const xcal_batch* bt, double* ms4) {
    if (!bt || !ms4) return XCAL_ERR_INVALID;
    for (int k = 0; k < 4; ++k) ms4[k] = bt->b->phase_ms[k];
    return XCAL_OK;
}

int32_t xcal_batch_case_index(const xcal_batch* bt, const xcal_case* cs, int32_t* index) {
    if (!bt || !cs || !index) return XCAL_ERR_INVALID;
    *index = bt->b->index_of(cs->c.get());
    return *index >= 0 ? XCAL_OK : XCAL_ERR_INVALID;
}

int32_t xcal_batch_simple_iterate(xcal_batch* bt, double* res, int32_t* converged) {
    if (!bt) return XCAL_ERR_INVALID;
    Batch* b = bt->b.get();
    XCAL_BGUARD(b->ctx, { b->simple_iteration(res, converged); })
}

}  // extern "C"
