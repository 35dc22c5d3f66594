// Serving: many tracking jobs of uneven size, algorithm, form and field map
// advanced together, tick by tick.
//
// ppt_jobs_create builds, in caller-provided device memory, the parameter
// block of every job (the same TrackDev / TrackMixDev the single-job kernels
// take), per-class work-queue index arrays, and per-job step counters and
// done flags.  ppt_jobs_tick then advances every unfinished job by up to
// `chunk` steps with one persistent kernel per (form, algorithm, RF, mixed
// map layout) class --
// blocks take (job, 128-particle block) items from a device queue -- followed
// by a one-thread-per-job kernel that advances the step counters.  The class
// kernels of a tick run concurrently: each is issued on a stream of its own
// that forks from the caller's stream and joins it again before the counter
// kernel (event dependencies, which a CUDA-graph capture records as parallel
// branches), so a class with few items no longer leaves the SMs idle while
// it drains.  A tick reads nothing from the host and synchronises nothing, so
// the host can capture it once per job set in a CUDA graph and replay it;
// jobs that finish simply find their done flag set on later replays.  No
// reference counterpart: the reference runs one track_batch call at a time
// (pusher.py:894-1012).
#include <cstring>
#include <mutex>
#include <vector>

#include "track_params.cuh"

struct ppt_jobs {
    int n_jobs;
    int device;
    struct Class {
        int precision;
        int algorithm;
        int rf;
        int layout;   // mixed form: the map's record layout
        int grid;
        ppt::JobQueueDev Q;
    };
    std::vector<Class> classes;
    std::vector<cudaStream_t> lanes;   // one stream per class (non-blocking), forked from the tick's stream
    std::vector<cudaEvent_t> joins;    // per lane: its class kernel is done
    cudaEvent_t fork = nullptr;        // the tick's stream reached the class kernels
    std::vector<char> image;   // host copy of the device table (kept for the upload's lifetime)
    unsigned* d_queues;
    int64_t* d_steps;
    int* d_done;
    const int64_t* d_total;
    const int64_t* d_window;
};

namespace ppt {

// classes: (form, algorithm, RF, record layout the job's kernel is
// specialised on; 0 = a float64 job's run-time dispatch over its maps)
constexpr int kLayouts[] = {kLayFull, kLayE, kLayB, kLayExEyBz, kLayEzBz, kLayBz, 0};
constexpr int kNumLayouts = 7;
constexpr int kMaxClasses = 2 * PPT_ALG_COUNT * 2 * kNumLayouts;

static int layout_index(int layout) {
    for (int i = 0; i < kNumLayouts; ++i)
        if (kLayouts[i] == layout) return i;
    return 0;
}

static size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

// Class lanes (a non-blocking stream and its join event) and fork events
// outlive the job tables that use them: a serving loop builds a table
// whenever its job set changes (tens of times a second), and creating and
// destroying a stream and an event per class each time cost more host time
// than the tick itself.  Destroyed tables return theirs here, per device;
// work still queued on a lane simply runs before the next table's.
struct LanePool {
    std::mutex mu;
    std::vector<std::vector<cudaStream_t>> streams;   // by device ordinal
    std::vector<std::vector<cudaEvent_t>> events;
};

static LanePool& lane_pool() {
    static LanePool* p = new LanePool();   // never destroyed: its streams live as long as the process
    return *p;
}

static cudaError_t take_stream(int dev, cudaStream_t* out) {
    LanePool& P = lane_pool();
    {
        std::lock_guard<std::mutex> g(P.mu);
        if ((int)P.streams.size() > dev && !P.streams[dev].empty()) {
            *out = P.streams[dev].back();
            P.streams[dev].pop_back();
            return cudaSuccess;
        }
    }
    return cudaStreamCreateWithFlags(out, cudaStreamNonBlocking);
}

static cudaError_t take_event(int dev, cudaEvent_t* out) {
    LanePool& P = lane_pool();
    {
        std::lock_guard<std::mutex> g(P.mu);
        if ((int)P.events.size() > dev && !P.events[dev].empty()) {
            *out = P.events[dev].back();
            P.events[dev].pop_back();
            return cudaSuccess;
        }
    }
    return cudaEventCreateWithFlags(out, cudaEventDisableTiming);
}

static void give_lanes(int dev, const std::vector<cudaStream_t>& streams, const std::vector<cudaEvent_t>& events) {
    LanePool& P = lane_pool();
    std::lock_guard<std::mutex> g(P.mu);
    if ((int)P.streams.size() <= dev) P.streams.resize(dev + 1);
    if ((int)P.events.size() <= dev) P.events.resize(dev + 1);
    P.streams[dev].insert(P.streams[dev].end(), streams.begin(), streams.end());
    P.events[dev].insert(P.events[dev].end(), events.begin(), events.end());
}

struct JobsLayout {
    size_t queues, steps, done, total, window, f64, mix, tindex, jindex, istart, bytes;
};

static JobsLayout jobs_layout(int n) {
    JobsLayout L;
    size_t o = 0;
    L.queues = o; o += al(sizeof(unsigned) * kMaxClasses);
    L.steps = o;  o += al(sizeof(int64_t) * n);
    L.done = o;   o += al(sizeof(int) * n);
    L.total = o;  o += al(sizeof(int64_t) * n);
    L.window = o; o += al(sizeof(int64_t) * n);
    L.f64 = o;    o += al(sizeof(TrackDev) * n);
    L.mix = o;    o += al(sizeof(TrackMixDev) * n);
    L.tindex = o; o += al(sizeof(int) * n);
    L.jindex = o; o += al(sizeof(int) * n);
    L.istart = o; o += al(sizeof(int) * (n + kMaxClasses));
    L.bytes = o;
    return L;
}

__global__ void jobs_advance_kernel(int n, int64_t* __restrict__ steps, int* __restrict__ done,
                                    const int64_t* __restrict__ total, const int64_t* __restrict__ window,
                                    int64_t chunk) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n || done[j]) return;
    const int64_t w = window[j] > 0 ? window[j] : chunk;
    int64_t k = total[j] - steps[j];
    if (k > w) k = w;
    steps[j] += k;
    if (steps[j] >= total[j]) done[j] = 1;
}

// Host-side parameter block of one job (same checks as ppt_track).
static int job_params(const ppt_job_desc& J, TrackDev* f64, TrackMixDev* mix) {
    int rc = check_state(&J.state);
    if (rc) return rc;
    if (J.nsteps_total < 0 || J.rec_every < 1) return fail(PPT_ERR_ARG, "job needs nsteps_total >= 0, rec_every >= 1");
    if ((J.r_hist == nullptr) != (J.v_hist == nullptr))
        return fail(PPT_ERR_ARG, "r_hist and v_hist must both be set or both be NULL");
    FieldsDev F;
    rc = build_fields(&J.fields, &F);
    if (rc) return rc;
    ppt_track_args a;
    std::memset(&a, 0, sizeof(a));
    a.nsteps_total = J.nsteps_total;
    a.rec_every = J.rec_every;
    a.dt = J.dt;
    a.q_over_m = J.q_over_m;
    a.t0 = J.t0;
    a.rf_omega = J.rf_omega;
    a.rf_phase = J.rf_phase;
    a.r_hist = J.r_hist;
    a.v_hist = J.v_hist;
    a.status = J.status;
    const int64_t n_rec = J.nsteps_total / J.rec_every + 1;
    if (J.state.precision == PPT_PREC_F64) {
        for (int i = 0; i < F.n_maps; ++i)
            if (F.maps[i].dtype != PPT_DTYPE_F64) return fail(PPT_ERR_ARG, "float64 jobs need float64 maps");
        std::memset(f64, 0, sizeof(*f64));
        f64->F = F;
        f64->n = J.state.n;
        f64->nsteps_total = J.nsteps_total;
        f64->rec_every = J.rec_every;
        f64->n_rec = n_rec;
        f64->dt = J.dt;
        f64->qm = J.q_over_m;
        f64->t0 = J.t0;
        f64->omega = J.rf_omega;
        f64->rf_phase = J.rf_phase;
        f64->f64 = J.state.f64;
        f64->r_hist = J.r_hist;
        f64->v_hist = J.v_hist;
        f64->status = J.status;
        return PPT_OK;
    }
    std::memset(mix, 0, sizeof(*mix));
    return make_track_mixed(F, &J.state, &a, n_rec, mix);
}

}  // namespace ppt

using namespace ppt;

extern "C" int64_t ppt_jobs_scratch_bytes(int n_jobs) {
    if (n_jobs < 0) return -1;
    return (int64_t)jobs_layout(n_jobs).bytes;
}

extern "C" int ppt_jobs_create(const ppt_job_desc* jobs, int n_jobs, void* scratch, ppt_jobs** out, void* stream) {
    if (!out) return fail(PPT_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (n_jobs < 0 || (n_jobs > 0 && !jobs)) return fail(PPT_ERR_ARG, "bad job list");
    if (!scratch) return fail(PPT_ERR_ARG, "scratch is NULL");
    const JobsLayout L = jobs_layout(n_jobs);
    ppt_jobs* H = new ppt_jobs();
    H->n_jobs = n_jobs;
    cudaGetDevice(&H->device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, H->device);
    H->image.assign(L.bytes, 0);
    char* img = H->image.data();
    char* dev = static_cast<char*>(scratch);
    TrackDev* f64 = reinterpret_cast<TrackDev*>(img + L.f64);
    TrackMixDev* mix = reinterpret_cast<TrackMixDev*>(img + L.mix);
    int64_t* total = reinterpret_cast<int64_t*>(img + L.total);
    int64_t* window = reinterpret_cast<int64_t*>(img + L.window);
    int* tindex = reinterpret_cast<int*>(img + L.tindex);
    int* jindex = reinterpret_cast<int*>(img + L.jindex);
    int* istart = reinterpret_cast<int*>(img + L.istart);
    // class of each job
    std::vector<int> cls(n_jobs);
    for (int j = 0; j < n_jobs; ++j) {
        int rc = job_params(jobs[j], f64 + j, mix + j);
        if (rc) {
            delete H;
            return rc;
        }
        total[j] = jobs[j].nsteps_total;
        if (jobs[j].steps_done < 0 || jobs[j].steps_done > jobs[j].nsteps_total) {
            delete H;
            return fail(PPT_ERR_ARG, "steps_done must be in [0, nsteps_total]");
        }
        if (jobs[j].tick_steps < 0 || jobs[j].tick_steps > 0x7fffffff) {
            delete H;
            return fail(PPT_ERR_ARG, "tick_steps must be in [0, 2^31)");
        }
        window[j] = jobs[j].tick_steps;
        reinterpret_cast<int64_t*>(img + L.steps)[j] = jobs[j].steps_done;
        const int rf = jobs[j].rf_phase != nullptr;
        const int lay = layout_index(jobs[j].state.precision == PPT_PREC_MIXED ? mix[j].map.layout
                                                                               : f64_single_layout(f64[j]));
        cls[j] = ((jobs[j].state.precision * PPT_ALG_COUNT + jobs[j].state.algorithm) * 2 + rf) * kNumLayouts + lay;
    }
    int pos = 0, ipos = 0;
    for (int c = 0; c < kMaxClasses; ++c) {
        const int first = pos;
        int items = 0;
        const int istart0 = ipos;
        for (int j = 0; j < n_jobs; ++j) {
            if (cls[j] != c) continue;
            tindex[pos] = j;
            jindex[pos] = j;
            istart[ipos++] = items;
            items += (int)((jobs[j].state.n + kJobBlock - 1) / kJobBlock);
            ++pos;
        }
        if (pos == first) continue;
        istart[ipos++] = items;
        ppt_jobs::Class K;
        const int c0 = c / kNumLayouts;
        K.precision = c0 / (2 * PPT_ALG_COUNT);
        K.algorithm = (c0 / 2) % PPT_ALG_COUNT;
        K.rf = c0 % 2;
        K.layout = kLayouts[c % kNumLayouts];
        K.grid = items < sms * 16 ? (items > 0 ? items : 1) : sms * 16;
        K.Q.table = dev + (K.precision == PPT_PREC_F64 ? L.f64 : L.mix);
        K.Q.table_index = reinterpret_cast<const int*>(dev + L.tindex) + first;
        K.Q.job_index = reinterpret_cast<const int*>(dev + L.jindex) + first;
        K.Q.item_start = reinterpret_cast<const int*>(dev + L.istart) + istart0;
        K.Q.n_jobs = pos - first;
        K.Q.n_items = items;
        K.Q.queue = reinterpret_cast<unsigned*>(dev + L.queues) + (int)H->classes.size();
        K.Q.steps = reinterpret_cast<const int64_t*>(dev + L.steps);
        K.Q.done = reinterpret_cast<const int*>(dev + L.done);
        K.Q.window = reinterpret_cast<const int64_t*>(dev + L.window);
        K.Q.chunk = 0;
        H->classes.push_back(K);
    }
    // one stream per class beyond the first, which runs on the caller's
    // stream (lanes and events from the device's pool)
    H->fork = nullptr;
    if (H->classes.size() > 1) {
        cudaError_t e = take_event(H->device, &H->fork);
        for (size_t i = 1; e == cudaSuccess && i < H->classes.size(); ++i) {
            cudaStream_t st;
            cudaEvent_t ev;
            e = take_stream(H->device, &st);
            if (e != cudaSuccess) break;
            H->lanes.push_back(st);
            e = take_event(H->device, &ev);
            if (e != cudaSuccess) break;
            H->joins.push_back(ev);
        }
        if (e != cudaSuccess) {
            ppt_jobs_destroy(H);
            return cuda_fail(e, "job class streams");
        }
    }
    H->d_queues = reinterpret_cast<unsigned*>(dev + L.queues);
    H->d_steps = reinterpret_cast<int64_t*>(dev + L.steps);
    H->d_done = reinterpret_cast<int*>(dev + L.done);
    H->d_total = reinterpret_cast<const int64_t*>(dev + L.total);
    H->d_window = reinterpret_cast<const int64_t*>(dev + L.window);
    cudaError_t e = cudaMemcpyAsync(scratch, img, L.bytes, cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        ppt_jobs_destroy(H);
        return cuda_fail(e, "job table upload");
    }
    *out = H;
    return PPT_OK;
}

extern "C" int ppt_jobs_tick(ppt_jobs* H, int64_t chunk, void* stream) {
    if (!H) return fail(PPT_ERR_ARG, "jobs handle is NULL");
    if (chunk < 0 || chunk > 0x7fffffff) return fail(PPT_ERR_ARG, "chunk must be in [0, 2^31)");
    if (H->n_jobs == 0) return PPT_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    PPT_CUDA_TRY(cudaMemsetAsync(H->d_queues, 0, sizeof(unsigned) * kMaxClasses, s));
    if (H->fork) PPT_CUDA_TRY(cudaEventRecord(H->fork, s));
    for (size_t i = 0; i < H->classes.size(); ++i) {
        const auto& K = H->classes[i];
        JobQueueDev Q = K.Q;
        Q.chunk = chunk;
        cudaStream_t cs = i == 0 ? s : H->lanes[i - 1];
        if (i > 0) PPT_CUDA_TRY(cudaStreamWaitEvent(cs, H->fork, 0));
        int rc = K.precision == PPT_PREC_F64 ? launch_f64_jobs(Q, K.algorithm, K.layout, K.rf != 0, K.grid, cs)
                                             : launch_mixed_jobs(Q, K.algorithm, K.layout, K.rf != 0, K.grid, cs);
        if (rc) return rc;
        if (i > 0) PPT_CUDA_TRY(cudaEventRecord(H->joins[i - 1], cs));
    }
    for (size_t i = 1; i < H->classes.size(); ++i) PPT_CUDA_TRY(cudaStreamWaitEvent(s, H->joins[i - 1], 0));
    jobs_advance_kernel<<<(H->n_jobs + 255) / 256, 256, 0, s>>>(H->n_jobs, H->d_steps, H->d_done, H->d_total,
                                                                H->d_window, chunk);
    PPT_CUDA_TRY(cudaGetLastError());
    return PPT_OK;
}

extern "C" int ppt_jobs_progress(const ppt_jobs* H, int64_t** steps, int32_t** done) {
    if (!H) return fail(PPT_ERR_ARG, "jobs handle is NULL");
    if (steps) *steps = H->d_steps;
    if (done) *done = H->d_done;
    return PPT_OK;
}

extern "C" int ppt_jobs_destroy(ppt_jobs* H) {
    if (!H) return PPT_OK;
    // lanes and events go back to the device's pool; work still queued on a
    // lane completes before anything a later table issues on it
    std::vector<cudaEvent_t> events(H->joins);
    if (H->fork) events.push_back(H->fork);
    give_lanes(H->device, H->lanes, events);
    delete H;
    return PPT_OK;
}
