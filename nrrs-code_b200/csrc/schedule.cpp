// schedule.cpp -- host-side control of the path: the per-depth strategy search (UBS) and the
// training schedule through steps 0-3. No GPU work.
//
// Replaces, in banbao990/NRRS-Code (NRRSPathTracer):
//   UBSUseNetOutputRRS / UBSNeedNetInfer / UBSUpdateAccordingArrayChar / UBSResetAndBeginSearch /
//   UBSEndSearch                      src/render/nrrs/integrator.h:324-405
//   isInferMode                       src/render/nrrs/integrator.h:67-71
//   UBSRecordEfficiency / UBSNextState / UBSAnalyseFrame
//                                     src/render/nrrs/integrator.cpp:2787-2891
//   autoTrainControl                  src/render/nrrs/integrator.cpp:2659-2736
// The search enumerates strategy strings as base-3 numbers, one digit per depth, and scores each
// by resolution / (frame time x error). It keeps the reference's stepping: the first 729 states
// (the lowest six digits) one by one, then, from the best state found so far, in steps of 729.
#include <cmath>
#include <cstring>
#include <new>

#include "nrrs.h"

namespace {

constexpr int kMaxDepthArray = 64;   // UBS_MAX_DEPTH (integrator.h:284)
constexpr int kStage = 729;          // 3^6

}  // namespace

struct nrrs_ubs {
    int max_depth = 6;
    double error_eval_seconds = 0.17e-3;
    bool search = false, use_best = false;
    int best_array[kMaxDepthArray] = {};
    float best_efficiency = -1.0f;
    int search_state = -1, search_state_mod = -1, last_search_state = -1;
    int max_state = 0, best_state = 0, stage = 0;
    bool timer_initialized = false;
    float last_error = -1.0f, last_delta_time = -1.0f;
    double last_time = 0.0;
};

struct nrrs_train_schedule {
    double state_end[5] = {};        // cumulative ends of states 0..3 (index 1..4)
    int state = -1;
    nrrs_train_schedule_state out{};
    int countdown = 100;
    double count_start = 0.0;
};

namespace {

int digit(int state, int depth) {
    int level = 1;
    for (int i = 0; i < depth; ++i) level *= NRRS_UBS_COUNT;
    return (state / level) % NRRS_UBS_COUNT;
}

// UBSResetAndBeginSearch (integrator.h:376-389)
void begin_search(nrrs_ubs* u) {
    u->best_efficiency = 0.0f;
    u->last_error = -1.0f;
    u->last_delta_time = -1.0f;
    u->search = true;
    u->use_best = false;
    u->search_state = -1;
    u->search_state_mod = -1;
    u->last_search_state = -1;
    u->max_state = (int)std::pow(3.0f, (float)u->max_depth);
}

// UBSEndSearch (integrator.h:391-405)
void end_search(nrrs_ubs* u) {
    u->timer_initialized = false;
    u->search = false;
    int s = u->best_state;
    for (int i = 0; i < u->max_depth; ++i) {
        u->best_array[i] = s % NRRS_UBS_COUNT;
        s /= NRRS_UBS_COUNT;
    }
}

}  // namespace

extern "C" int nrrs_ubs_create(int32_t max_depth, double error_eval_seconds, nrrs_ubs** out) {
    if (!out || max_depth < 1 || max_depth > 19 || !(error_eval_seconds >= 0.0))
        return NRRS_ERR_INVALID_ARG;
    nrrs_ubs* u = new (std::nothrow) nrrs_ubs();
    if (!u) return NRRS_ERR_INVALID_ARG;
    u->max_depth = max_depth;
    u->error_eval_seconds = error_eval_seconds;
    *out = u;
    return NRRS_OK;
}

extern "C" void nrrs_ubs_destroy(nrrs_ubs* u) { delete u; }

extern "C" int nrrs_ubs_begin_search(nrrs_ubs* u) {
    if (!u) return NRRS_ERR_INVALID_ARG;
    begin_search(u);
    return NRRS_OK;
}

// UBSNextState (integrator.cpp:2798-2820), and UBSEndSearch once it returns false
// (render(), integrator.cpp:1780-1783)
extern "C" int nrrs_ubs_next_state(nrrs_ubs* u) {
    if (!u) return NRRS_ERR_INVALID_ARG;
    if (!u->search) return 0;
    if (u->search_state < u->max_state) {
        u->last_search_state = u->search_state;
        if (u->search_state == 0) u->stage = 0;
        ++u->search_state_mod;
        if (u->search_state_mod == kStage) {
            ++u->stage;
            u->search_state = u->best_state;
        }
        int step = 1;
        for (int i = 0; i < u->stage; ++i) step *= kStage;
        u->search_state += step;
        return 1;
    }
    end_search(u);
    return 0;
}

// UBSAnalyseFrame (integrator.cpp:2822-2889) without the kernels: the caller brings its clock
// and the frame's error sum, which stands for the value the reference copies back
// asynchronously and reads at the next call.
extern "C" int nrrs_ubs_analyse_frame(nrrs_ubs* u, double now_seconds, double frame_error_sum,
                                      uint32_t resolution) {
    if (!u) return NRRS_ERR_INVALID_ARG;
    if (!u->search) return NRRS_OK;
    if (!u->timer_initialized) {
        begin_search(u);
        u->timer_initialized = true;
        u->last_time = now_seconds;
        return NRRS_OK;
    }
    const float delta = (float)(now_seconds - u->last_time);
    u->last_time = now_seconds;
    if (u->last_error < 0.0f) {
        const int keep = u->last_search_state;   // first attempt: restart, keep the state
        begin_search(u);
        u->last_search_state = keep;
    } else if (u->last_search_state >= 0) {
        u->last_delta_time -= (float)u->error_eval_seconds;
        const float eff = (float)resolution / (u->last_delta_time * u->last_error);
        if (eff > u->best_efficiency) {           // UBSRecordEfficiency (:2787-2796)
            u->best_efficiency = eff;
            u->best_state = u->last_search_state;
        }
    }
    u->last_delta_time = delta;
    u->last_error = (float)frame_error_sum;
    return NRRS_OK;
}

extern "C" int nrrs_ubs_get_strategy(const nrrs_ubs* u, int32_t depth) {
    if (!u || depth < 0 || depth >= kMaxDepthArray) return NRRS_ERR_INVALID_ARG;
    if (u->search) return digit(u->search_state, depth);
    if (u->use_best) return u->best_array[depth];
    return -1;
}

// isInferMode (integrator.h:67-71) with UBSNeedNetInfer (:348-362), and the factor source of
// generateRRSNumber (integrator.cpp:1088-1090) with UBSUseNetOutputRRS (:324-346)
extern "C" int nrrs_ubs_need_infer(const nrrs_ubs* u, int32_t depth, int32_t enable_rrs,
                                   float clamp_min, float clamp_max, int32_t max_rrs_depth,
                                   int32_t use_net_output_rrs, int32_t* factor_source) {
    if (!u || depth < 0 || depth >= kMaxDepthArray) return NRRS_ERR_INVALID_ARG;
    bool need = true;
    if (u->use_best) need = u->best_array[depth] != NRRS_UBS_FIXED_RR;
    else if (u->search) need = digit(u->search_state, depth) != NRRS_UBS_FIXED_RR;
    const bool infer = enable_rrs && clamp_min < clamp_max && depth <= max_rrs_depth && need;
    if (factor_source) {
        bool net = use_net_output_rrs != 0;
        if (u->search) net = digit(u->search_state, depth) == NRRS_UBS_NRRS;
        else if (u->use_best) net = u->best_array[depth] == NRRS_UBS_NRRS;
        *factor_source = net ? NRRS_FACTOR_RRSNET : NRRS_FACTOR_ADRRS;
    }
    return infer ? 1 : 0;
}

extern "C" int nrrs_ubs_best(const nrrs_ubs* u, int32_t* strategy, float* efficiency) {
    if (!u) return NRRS_ERR_INVALID_ARG;
    if (strategy)
        for (int i = 0; i < u->max_depth; ++i) strategy[i] = u->best_array[i];
    if (efficiency) *efficiency = u->best_efficiency;
    return NRRS_OK;
}

// UBSUpdateAccordingArrayChar (integrator.h:364-374); the reference's UI then ticks
// "Use Best Strategy" (integrator.cpp:2181)
extern "C" int nrrs_ubs_set_best(nrrs_ubs* u, const char* digits) {
    if (!u || !digits) return NRRS_ERR_INVALID_ARG;
    const size_t len = std::strlen(digits);
    for (int i = 0; i < u->max_depth; ++i) {
        const int num = i < (int)len ? digits[i] - '0' : -1;
        u->best_array[i] = (num >= 0 && num < NRRS_UBS_COUNT) ? num : NRRS_UBS_FIXED_RR;
    }
    u->use_best = true;
    return NRRS_OK;
}

extern "C" int nrrs_ubs_searching(const nrrs_ubs* u) { return u && u->search ? 1 : 0; }

extern "C" int nrrs_train_schedule_create(const double durations[4], nrrs_train_schedule** out) {
    if (!out || !durations) return NRRS_ERR_INVALID_ARG;
    nrrs_train_schedule* s = new (std::nothrow) nrrs_train_schedule();
    if (!s) return NRRS_ERR_INVALID_ARG;
    for (int i = 1; i < 5; ++i) {
        if (!(durations[i - 1] >= 0.0)) { delete s; return NRRS_ERR_INVALID_ARG; }
        s->state_end[i] = s->state_end[i - 1] + durations[i - 1];
    }
    *out = s;
    return NRRS_OK;
}

extern "C" void nrrs_train_schedule_destroy(nrrs_train_schedule* s) { delete s; }

// autoTrainControl (integrator.cpp:2659-2736); like the reference, one tick may pass through
// several states whose time is already over
extern "C" int nrrs_train_schedule_tick(nrrs_train_schedule* s, double elapsed, double now_seconds,
                                        nrrs_train_schedule_state* out) {
    if (!s || !out) return NRRS_ERR_INVALID_ARG;
    nrrs_train_schedule_state& o = s->out;
    auto over = [&](int st) { return elapsed > s->state_end[st + 1]; };
    if (s->state == -1) {
        s->state = 0;
        o.enable_rrs = 0;
        o.step = 0;
    }
    if (s->state == 0 && over(0)) {
        s->state = 1;
        o.enable_rrs = 0;
        o.step = 1;
    }
    if (s->state == 1 && over(1)) {
        s->state = 2;
        o.enable_rrs = 1;
        o.use_net_output_rrs = 0;
        o.step = 2;
    }
    if (s->state == 2 && over(2)) {
        s->state = 3;
        o.use_net_output_rrs = 1;
        o.step = 3;
    }
    if (s->state == 3 && over(3)) {
        o.stop_training = 1;
        if (s->countdown == 100) s->count_start = now_seconds;
        if (--s->countdown < 0) {
            o.seconds_per_frame = (now_seconds - s->count_start) / 100.0;
            s->state = 4;
        }
    }
    if (s->state == 4) o.request_exit = 1;
    o.state = s->state;
    *out = o;
    return NRRS_OK;
}
