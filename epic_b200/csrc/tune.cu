// Autotuner: picks the launch shapes of one context by timing the candidates
// on its own parcels and grid.  Only calls whose results do not depend on the
// choice and that leave the simulation state as it was are timed: par2grid
// and vol2grid with the support vectors recomputed (the same values are
// stored again) and forward horizontal FFTs of a field into work arrays.
#include "ctx.hpp"

#include <algorithm>
#include <cfloat>

namespace epic {

template <class F>
static float time_ms(Ctx& c, F&& run, int reps = 3) {
    struct Events {   // destroyed on every exit, an error in run() included
        cudaEvent_t e[2] = {nullptr, nullptr};
        ~Events() {
            for (cudaEvent_t x : e)
                if (x) cudaEventDestroy(x);
        }
    } ev;
    CK(cudaEventCreate(&ev.e[0]));
    CK(cudaEventCreate(&ev.e[1]));
    cudaEvent_t a = ev.e[0], b = ev.e[1];
    run();   // warm-up (module load, caches)
    float best = FLT_MAX;
    for (int r = 0; r < reps; ++r) {
        CK(cudaEventRecord(a, c.stream));
        run();
        CK(cudaEventRecord(b, c.stream));
        CK(cudaEventSynchronize(b));
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, a, b));
        best = std::min(best, ms);
    }
    return best;
}

void autotune(Ctx& c, epic_tuning* out) {
    if (!c.has_parcels || c.n == 0) throw CudaError(EPIC_ERR_STATE, "autotune: no parcels");
    // time the box-ordered paths the steps use (the parcel set is unchanged)
    if (!c.cfg.keep_order) sort_parcels(c);
    // lane groups of the par2grid scatter (also the stage's par2grid) and of vol2grid
    int best_p = c.scatter_lg[1], best_v = c.scatter_lg[0];
    float tp = FLT_MAX, tv = FLT_MAX;
    for (int lg = 0; lg <= 3; ++lg) {
        c.scatter_lg[1] = lg;
        float t = time_ms(c, [&] { par2grid(c, false, true); });
        if (t < tp) { tp = t; best_p = lg; }
        c.scatter_lg[0] = lg;
        t = time_ms(c, [&] { vol2grid(c, false); });
        if (t < tv) { tv = t; best_v = lg; }
    }
    c.scatter_lg[1] = c.scatter_lg[2] = best_p;
    c.scatter_lg[0] = best_v;
    // horizontal FFT path: plane kernel (square grids up to 128), tiled lines, Stockham lines,
    // half-plane cluster kernel (square 64 and 128)
    int best_f = c.fft_path;
    float tf = FLT_MAX;
    for (int path = 0; path <= 3; ++path) {
        c.fft_path = path;
        float t = time_ms(c, [&] { fft_forward_probe(c); });
        if (t < tf) { tf = t; best_f = path; }
    }
    c.fft_path = best_f;
    // leave the fields as a plain par2grid would (the probes overwrote work arrays only)
    par2grid(c, false, true);
    CK(cudaStreamSynchronize(c.stream));
    if (out) {
        out->lg_par2grid = best_p;
        out->lg_vol2grid = best_v;
        out->fft_path = best_f;
        out->ms_par2grid = tp;
        out->ms_vol2grid = tv;
        out->ms_fft = tf;
    }
}

}  // namespace epic
