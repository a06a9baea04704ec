// Host-side harness around reference code, built from the reference checkout by oracle/Makefile
// into oracle/_ref/ (test infrastructure: it pins the oracle's restatements; the product library
// never sees it). What is compiled, from the reference's own sources:
//   RRSWeightWindow             src/render/common/commoncudautils.h:14-28   (its own header)
//   activationSigma             src/render/nrrs/net/networkcommon.h:61-68   (its own header; its
//                               KiRaRay and tiny-cuda-nn includes resolve to oracle/ref_stubs)
//   warp_roughness              src/render/nrrs/train.h:95                  (function text)
//   box_cox_transform (scalar)  src/render/nrrs/train.cu:19-28              (function text)
//   "Gen RRS Number" lambda     src/render/nrrs/integrator.cpp:1186-1297    (lambda text)
//   "Gen Tids" lambda           src/render/nrrs/integrator.cpp:1370-1457    (lambda text)
// The Makefile copies the function and lambda texts, at build time, from the reference files
// into oracle/_ref/gen (extract_block.awk); nothing of them is stored in the repository.
//
// Each lambda runs once per vertex, in vertex order, over stand-ins of the integrator members it
// reads. The stand-ins below replace KiRaRay types and helpers that are absent from the
// checkout (its submodule is empty): RGB with Eigen-style element-wise operators and
// mean() = (r + g + b) / 3, clamp = min(max(x, lo), hi) per element, the sampler's get1D (which
// returns the given rnd of the vertex), and TidQueue::push(tid, cnt), which appends cnt copies
// of tid (commonworkqueue.h:19-25; sequential here, so the queue is in vertex order).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "render/common/commoncudautils.h"
#include "render/nrrs/net/networkcommon.h"

namespace refh {

struct RGB {
    float v[3];
    RGB() : v{0.f, 0.f, 0.f} {}
    explicit RGB(float x) : v{x, x, x} {}
    RGB(float a, float b, float c) : v{a, b, c} {}
    float operator[](int k) const { return v[k]; }
    float& operator[](int k) { return v[k]; }
    float mean() const { return (v[0] + v[1] + v[2]) / 3.0f; }
};
inline RGB operator*(const RGB& a, const RGB& b) { return RGB(a[0] * b[0], a[1] * b[1], a[2] * b[2]); }
inline RGB operator/(const RGB& a, const RGB& b) { return RGB(a[0] / b[0], a[1] / b[1], a[2] / b[2]); }
inline RGB operator/(const RGB& a, float s) { return RGB(a[0] / s, a[1] / s, a[2] / s); }
inline RGB operator+(const RGB& a, float s) { return RGB(a[0] + s, a[1] + s, a[2] + s); }
inline float clamp(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }
inline RGB clamp(const RGB& a, float lo, float hi) {
    return RGB(clamp(a[0], lo, hi), clamp(a[1], lo, hi), clamp(a[2], lo, hi));
}
inline float atomicAdd(float* p, float x) { const float o = *p; *p += x; return o; }
// CUDA's math headers give device code float overloads of the C math functions, so the
// reference's sqrt(x) on a float x is a float square root on the GPU; a host build would pick
// C's double sqrt instead. The overload restores the device meaning for the compiled texts.
inline float sqrt(float x) { return std::sqrt(x); }
inline uint32_t offsetFrame2Scaled(uint32_t pixel, int, uint32_t) { return pixel; }

struct ColorSpace {};
struct AnyArg {};
inline ColorSpace g_colorspace;
struct ThpItem {
    RGB c;
    RGB toRGB(AnyArg, const ColorSpace&) const { return c; }
    ThpItem& operator=(const RGB& x) { c = x; return *this; }
};
struct Pixel {
    RGB c;
    template <int N> RGB head() const { return c; }
};
struct Film {
    const RGB* px;
    Pixel getPixel(uint32_t i) const { return Pixel{px[i]}; }
};
struct InferenceQueue { const uint32_t* mScatterQueueIndex; };
struct Sampler {
    float r;
    float get1D() { return r; }
};
struct PixelState { Sampler* mSampler; };
struct IntrSoa {
    const RGB* p;
    const RGB* wo;
    struct { const float* roughness; } sd;
};
struct ScatterRayQueue {
    float* mRRS;
    const uint32_t* mPixelId;
    int* mNodeIdx;
    IntrSoa mIntr;
};
struct PathState {
    template <typename... A> int recordNode(A...) { return -1; }
};
struct TidQueue {
    std::vector<uint32_t> q;
    void push(uint32_t tid, int cnt) { for (int k = 0; k < cnt; ++k) q.push_back(tid); }
};

}  // namespace refh

#define KRR_DEVICE_LAMBDA(...) [&](__VA_ARGS__)
#define KRR_DEFAULT_COLORSPACE_GPU (&refh::g_colorspace)

namespace refh {
using krr::activationSigma;
using precision_t = float;
constexpr uint32_t NRRS_LL2NET_DIM_OUTPUT_PADDED = 16;
constexpr uint32_t NRRS_RRSNET_DIM_OUTPUT_PADDED = 16;

#include "gen/warp_roughness.inc"
#include "gen/box_cox.inc"
}  // namespace refh

extern "C" float ref_rrs_weight_window(float x, float ww) { return RRSWeightWindow(x, ww); }
extern "C" float ref_activation_sigma(float x) { return krr::activationSigma(x); }
extern "C" float ref_warp_roughness(float r) { return refh::warp_roughness(r); }
extern "C" float ref_box_cox(float x) { return refh::box_cox_transform(x); }

// "Gen RRS Number" for n vertices. net_out is [n][16] as the networks write it: RRSNet's raw
// factor at [i][0] (use_network = 1) or StatNet's L at [i][0..2] (use_network = 0, ADRRS);
// thp and ref_rgb are [n][3] (the vertex throughput and its pixel's rendered colour).
// rrs[n] and rrs_ceil[n] receive the clamped factor and its ceiling.
extern "C" void ref_gen_rrs_number(uint32_t n, int use_network, const float* net_out,
                                   const float* thp, const float* ref_rgb, int use_ww,
                                   float clamp_min, float clamp_max, int use_ceil, float* rrs_out,
                                   float* rrs_ceil_out) {
    using namespace refh;
    std::vector<uint32_t> ident(n);
    for (uint32_t i = 0; i < n; ++i) ident[i] = i;
    std::vector<ThpItem> thp_items(n);
    std::vector<RGB> ref_px(n);
    for (uint32_t i = 0; i < n; ++i) {
        thp_items[i].c = RGB(thp[3 * i], thp[3 * i + 1], thp[3 * i + 2]);
        ref_px[i] = RGB(ref_rgb[3 * i], ref_rgb[3 * i + 1], ref_rgb[3 * i + 2]);
    }
    InferenceQueue iq{ident.data()};
    InferenceQueue* mInferenceQueue = &iq;
    auto getPixelIdArray = [&]() { return ident.data(); };
    auto getThpArray = [&]() { return thp_items.data(); };
    Film film{ref_px.data()};
    Film* mRenderedImage = &film;
    const RGB* mRenderedImageDenoised = ref_px.data();
    const bool mUseTheAccmulatedBufferInsteadOfTheDenosiedBuffer = true;
    const uint32_t mErrorImageScale = 1;
    const bool useNetworkOutputRRS = use_network != 0;
    const precision_t* outputDataPtr = net_out;
    const bool mRRSDivInRect = false;
    std::vector<Sampler> samplers(n, Sampler{0.f});
    PixelState ps{samplers.data()};
    PixelState* mPixelState = &ps;
    const int frameSize[2] = {(int)n, 1};
    const int drawCenter[2] = {0, 0};
    const int mDrawRectSize = 0;
    const float mRRSDivInRectVal = 1.f;
    const bool mDebugTrainingData = false;
    const int mDebugPixel = -1;
    const int depth = 0;
    const bool useWeightWindow = use_ww != 0;
    const float RRS_CLAMP_MIN = clamp_min, RRS_CLAMP_MAX = clamp_max;
    const bool updateShowRRSBuffer0 = false, updateShowRRSBuffer1 = false;
    float* showRRSBuffer = nullptr;
    float* rrsArray = rrs_out;
    float* rrsArrayCeil = rrs_ceil_out;
    const bool useCeil = use_ceil != 0;
    auto body =
#include "gen/gen_rrs_number.inc"
        ;
    for (uint32_t tid = 0; tid < n; ++tid) body((int)tid);
}

// "Gen Tids" for n vertices: rrs_in[n] are the clamped factors, rnd[n] the sampler's draws,
// rcp_sum the reciprocal of the normalisation sum, budget the pixel count, n_specular the
// specular count. rrs_norm[n] receives mScatterRayQueue->mRRS; queue (capacity entries)
// receives the pushed scatter indices. Returns the queue size (beyond capacity: not written).
extern "C" uint64_t ref_gen_tids(uint32_t n, const float* rrs_in, const float* rnd,
                                 uint32_t budget, uint32_t n_specular, float rcp_sum,
                                 int use_ceil, float normalize_rate, int scale_up,
                                 float* rrs_norm, uint32_t* queue, uint64_t capacity) {
    using namespace refh;
    constexpr bool tIsSimpleMode = false;
    constexpr bool tIsTraining = false;
    std::vector<uint32_t> ident(n);
    for (uint32_t i = 0; i < n; ++i) ident[i] = i;
    std::vector<ThpItem> thp_items(n);
    InferenceQueue iq{ident.data()};
    InferenceQueue* mInferenceQueue = &iq;
    auto getThpArray = [&]() { return thp_items.data(); };
    auto getPixelIdArray = [&]() { return ident.data(); };
    const uint32_t resolutionSize = budget;
    const uint32_t spec = n_specular;
    const uint32_t* specularSize = &spec;
    const float* rrsSumRcp = &rcp_sum;
    const bool useCeil = use_ceil != 0;
    const float RRS_NORMALIZE_RATE = normalize_rate;
    const bool printNormalizeFactor = false;
    const int depth = 0;
    const bool mDebugRRSNormalized = false;
    const bool shouldScaleUp = scale_up != 0;
    const float* rrsArray = rrs_in;
    std::vector<int> node_idx(n, -1);
    ScatterRayQueue srq{rrs_norm, ident.data(), node_idx.data(), IntrSoa{nullptr, nullptr, {nullptr}}};
    ScatterRayQueue* mScatterRayQueue = &srq;
    std::vector<Sampler> samplers(n);
    for (uint32_t i = 0; i < n; ++i) samplers[i].r = rnd[i];
    PixelState ps{samplers.data()};
    PixelState* mPixelState = &ps;
    const bool copyTheRRSNode = true;
    PathState pstate;
    PathState* mPathState = &pstate;
    const bool updateShowRRSBuffer2 = false, updateShowRRSBuffer3 = false;
    float* showRRSBuffer = nullptr;
    TidQueue tq;
    TidQueue* mScatterTidQueue = &tq;
    auto body =
#include "gen/gen_tids.inc"
        ;
    for (uint32_t tid = 0; tid < n; ++tid) body((int)tid);
    for (uint64_t k = 0; k < tq.q.size() && k < capacity; ++k) queue[k] = tq.q[k];
    return tq.q.size();
}
