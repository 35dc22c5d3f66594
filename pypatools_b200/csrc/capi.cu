// extern "C" entry points: argument checks, parameter blocks, dispatch to the
// float64 or mixed-precision track kernels, error strings.
#include <cstring>
#include <string>

#include "track_params.cuh"

namespace ppt {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t err, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(err);
    return PPT_ERR_CUDA;
}

static int check_track_args(const ppt_state* st, const ppt_track_args* a) {
    if (!a) return fail(PPT_ERR_ARG, "track args are NULL");
    if (a->nsteps < 0 || a->step0 < 0) return fail(PPT_ERR_ARG, "step0 and nsteps must be >= 0");
    if (a->nsteps > 0x7fffffff) return fail(PPT_ERR_ARG, "nsteps per call must fit int32");
    if (a->rec_every < 1) return fail(PPT_ERR_ARG, "rec_every must be >= 1");
    if (a->nsteps_total < a->step0 + a->nsteps) return fail(PPT_ERR_ARG, "nsteps_total < step0 + nsteps");
    if ((a->r_hist == nullptr) != (a->v_hist == nullptr))
        return fail(PPT_ERR_ARG, "r_hist and v_hist must both be set or both be NULL");
    if (!(a->dt == a->dt)) return fail(PPT_ERR_ARG, "dt is NaN");
    if ((a->flags & ~(PPT_TRACK_INIT | PPT_TRACK_FINAL)) != 0) return fail(PPT_ERR_ARG, "unknown track flags");
    (void)st;
    return PPT_OK;
}

}  // namespace ppt

using namespace ppt;

extern "C" const char* ppt_last_error(void) { return g_last_error.c_str(); }

extern "C" int ppt_abi_version(void) { return PPT_ABI_VERSION; }

extern "C" int ppt_track(ppt_state* st, const ppt_fields* fields, const ppt_track_args* a, void* stream) {
    int rc = check_state(st);
    if (rc) return rc;
    rc = check_track_args(st, a);
    if (rc) return rc;
    if (st->n == 0 || (a->nsteps == 0 && !(a->flags & (PPT_TRACK_INIT | PPT_TRACK_FINAL)))) return PPT_OK;
    FieldsDev F;
    rc = build_fields(fields, &F);
    if (rc) return rc;
    const int64_t n_rec = a->nsteps_total / a->rec_every + 1;
    const bool rf = a->rf_phase != nullptr;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (st->precision == PPT_PREC_F64) {
        for (int i = 0; i < F.n_maps; ++i)
            if (F.maps[i].dtype != PPT_DTYPE_F64)
                return fail(PPT_ERR_ARG, "the float64 form needs float64 maps (create them with PPT_DTYPE_F64)");
        TrackDev P;
        std::memset(&P, 0, sizeof(P));
        P.F = F;
        P.n = st->n;
        P.step0 = a->step0;
        P.nsteps = a->nsteps;
        P.nsteps_total = a->nsteps_total;
        P.rec_every = a->rec_every;
        P.n_rec = n_rec;
        P.flags = a->flags;
        P.dt = a->dt;
        P.qm = a->q_over_m;
        P.t0 = a->t0;
        P.omega = a->rf_omega;
        P.rf_phase = a->rf_phase;
        P.f64 = st->f64;
        P.r_hist = a->r_hist;
        P.v_hist = a->v_hist;
        P.order = a->order;
        P.status = a->status;
        P.counters = a->counters;
        if (a->surface) {
            if (!a->active) return fail(PPT_ERR_ARG, "a surface needs the active array");
            P.surf = a->surface->dev;
            P.active = a->active;
        }
        if (a->dt_rows) {
            // the reference's batch RK4 step is the one that broadcasts an array dt
            // (pusher.py:815-816); its other pushers take a float
            if (st->algorithm != PPT_ALG_RK4 && st->algorithm != PPT_ALG_RK4_REL)
                return fail(PPT_ERR_UNSUPPORTED, "a per-particle dt needs the rk4 or rk4_rel algorithm");
            P.dt_rows = a->dt_rows;
        }
        // the launch's per-step RF table covers steps step0 .. step0 + nsteps
        // (the closing half step reads the last one); a per-particle dt has none
        P.rf_tab_n = (rf && !a->dt_rows && a->nsteps + 1 <= 512) ? (int32_t)(a->nsteps + 1) : 0;
        return launch_track_f64(P, st->algorithm, rf, a->surface != nullptr, s);
    }
    if (a->dt_rows) return fail(PPT_ERR_UNSUPPORTED, "a per-particle dt runs in the float64 form");
    if (a->surface && st->algorithm != PPT_ALG_BORIS)
        return fail(PPT_ERR_UNSUPPORTED, "electrode surfaces run in the float64 form and the mixed form's boris");
    if (a->surface && !a->active) return fail(PPT_ERR_ARG, "a surface needs the active array");
    TrackMixDev P;
    std::memset(&P, 0, sizeof(P));
    rc = make_track_mixed(F, st, a, n_rec, &P);
    if (rc) return rc;
    if (a->surface) {
        CollDev C;
        C.surf = a->surface->dev;
        C.active = a->active;
        return launch_track_mixed_coll(P, C, rf, s);
    }
    return launch_track_mixed(P, st->algorithm, rf, s);
}
