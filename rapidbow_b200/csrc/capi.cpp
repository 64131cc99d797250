// extern "C" entry points (include/rapidbow_b200.h).  Exceptions stop here: every entry point
// returns an rbw_status and leaves a message for rbw_last_error().
#include "rapidbow_b200.h"
#include "vocabulary.h"
#include "timing.h"
#include "tuning.h"
#include "capi_internal.h"

#include <cstring>
#include <new>
#include <string>

struct rbw_vocabulary {
    std::unique_ptr<rbw::Vocabulary> v;
};

namespace {
thread_local std::string gLastError;

template <typename F>
int guard(F&& f)
{
    try {
        f();
        return RBW_OK;
    } catch (const rbw::Error& e) {
        gLastError = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        gLastError = "host allocation failed";
        return RBW_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        gLastError = e.what();
        return RBW_ERR_INTERNAL;
    }
}

void requireSift(const rbw_desc_attr& a)
{
    if (a.data_type != RBW_DATA_UINT8 || a.distance_type != RBW_DIST_L2 || a.nb_dims != 128) {
        // RapidBoW.cpp:37-39
        throw rbw::Error(rbw::kUnsupported,
                         "Only {DataType::kUInt8, DistanceType::kL2, 128}, i.e. quantized SIFT, is supported");
    }
}

const rbw::Vocabulary& vocOf(const rbw_vocabulary* h)
{
    if (h == nullptr || !h->v) throw rbw::Error(rbw::kInvalidArg, "null vocabulary handle");
    return *h->v;
}
} // namespace

extern "C" {

const char* rbw_last_error(void) { return gLastError.c_str(); }

const char* rbw_version(void) { return "rapidbow_b200 0.1.0 (sm_100a)"; }

void rbw_build_options_default(rbw_build_options* o)
{
    if (o == nullptr) return;
    std::memset(o, 0, sizeof(*o));
    o->max_iterations = 1000;
    o->check_interval = 4;
    o->init_mode = RBW_INIT_REFERENCE;
}

int rbw_voc_build(rbw_desc_attr attr, uint32_t branch_factor, const void* dev_desc, uint32_t nb_desc, uint32_t nb_doc,
                  uint32_t nb_levels, const rbw_build_options* opts, void* stream, rbw_vocabulary** out)
{
    return guard([&] {
        if (out == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output handle");
        *out = nullptr;
        requireSift(attr);
        rbw::BuildOptions o{};
        if (opts != nullptr) {
            o.maxIterations = opts->max_iterations;
            o.checkInterval = opts->check_interval;
            o.initMode = opts->init_mode;
            o.seed = opts->seed;
            o.injected = opts->injected_init;
            o.ieeeDivision = (opts->flags & RBW_BUILD_IEEE_DIVISION) != 0;
            o.floatCenters = (opts->flags & RBW_BUILD_FLOAT_CENTERS) != 0;
            if (opts->flags & ~uint32_t(RBW_BUILD_IEEE_DIVISION | RBW_BUILD_FLOAT_CENTERS))
                throw rbw::Error(rbw::kInvalidArg, "unknown build flag");
            if (o.initMode > rbw::kInitInjected) throw rbw::Error(rbw::kInvalidArg, "unknown init mode");
        }
        auto v = rbw::Vocabulary::build(branch_factor, nb_levels, static_cast<const uint8_t*>(dev_desc), nb_desc,
                                        nb_doc, o, static_cast<cudaStream_t>(stream), nullptr);
        *out = new rbw_vocabulary{std::move(v)};
    });
}

int rbw_voc_from_host(uint32_t branch_factor, uint32_t nb_levels, const uint8_t* centers, const uint32_t* masks,
                      const float* weights, rbw_vocabulary** out)
{
    return guard([&] {
        if (out == nullptr || centers == nullptr || masks == nullptr || weights == nullptr)
            throw rbw::Error(rbw::kInvalidArg, "null argument");
        *out = nullptr;
        auto v = rbw::Vocabulary::fromHost(branch_factor, nb_levels, centers, masks, weights);
        *out = new rbw_vocabulary{std::move(v)};
    });
}

int rbw_voc_from_host_f32(uint32_t branch_factor, uint32_t nb_levels, const float* centers, const uint32_t* masks,
                          const float* weights, rbw_vocabulary** out)
{
    return guard([&] {
        if (out == nullptr || centers == nullptr || masks == nullptr || weights == nullptr)
            throw rbw::Error(rbw::kInvalidArg, "null argument");
        *out = nullptr;
        auto v = rbw::Vocabulary::fromHostF32(branch_factor, nb_levels, centers, masks, weights);
        *out = new rbw_vocabulary{std::move(v)};
    });
}

int rbw_voc_center_type(const rbw_vocabulary* voc, int32_t* type)
{
    return guard([&] {
        if (type == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output");
        *type = vocOf(voc).floatCenters() ? RBW_CENTERS_FLOAT32 : RBW_CENTERS_UINT8;
    });
}

int rbw_voc_get_centers_f32(const rbw_vocabulary* voc, float* host_centers)
{
    return guard([&] {
        if (host_centers == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output");
        const auto c = vocOf(voc).centersF32Host();
        std::memcpy(host_centers, c.data(), c.size() * sizeof(float));
    });
}

int rbw_voc_build_stats(const rbw_vocabulary* voc, rbw_build_stats* stats)
{
    return guard([&] {
        if (stats == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output");
        const rbw::BuildStats& s = vocOf(voc).buildStats();
        std::memset(stats, 0, sizeof(*stats));
        stats->levels = s.levels;
        for (int i = 0; i < 16; i++) {
            stats->iterations[i] = s.iterations[i];
            stats->inertia_first[i] = s.inertiaFirst[i];
            stats->inertia_last[i] = s.inertiaLast[i];
            stats->refined[i] = s.refined[i];
            stats->assignments[i] = s.assignments[i];
        }
        stats->seconds = s.seconds;
    });
}

int rbw_voc_refined_lookups(const rbw_vocabulary* voc, uint64_t* refined)
{
    return guard([&] {
        if (refined == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output");
        RBW_CUDA(cudaDeviceSynchronize());
        *refined = vocOf(voc).takeRefinedLookups();
    });
}

int rbw_voc_lookup(const rbw_vocabulary* voc, const void* dev_desc, uint32_t nb_desc, uint32_t* dev_leaf, void* stream)
{
    return guard([&] {
        vocOf(voc).lookup(static_cast<const uint8_t*>(dev_desc), nb_desc, dev_leaf, rbw::kLookupAuto,
                          static_cast<cudaStream_t>(stream));
    });
}

int rbw_voc_lookup_ex(const rbw_vocabulary* voc, const void* dev_desc, uint64_t nb_desc, uint32_t* dev_leaf,
                      int32_t algo, void* stream, uint32_t* kernels_launched)
{
    return guard([&] {
        if (algo < 0 || algo > rbw::kLookupAlgoLast)
            throw rbw::Error(rbw::kInvalidArg, "unknown lookup algorithm");
        const uint32_t k = vocOf(voc).lookup(static_cast<const uint8_t*>(dev_desc), nb_desc, dev_leaf,
                                             static_cast<rbw::LookupAlgo>(algo), static_cast<cudaStream_t>(stream));
        if (kernels_launched) *kernels_launched = k;
    });
}

int rbw_voc_lookup_host(const rbw_vocabulary* voc, const void* host_desc, uint64_t nb_desc, uint32_t* host_leaf,
                        int32_t algo, uint32_t* kernels_launched)
{
    return guard([&] {
        if (algo < 0 || algo > rbw::kLookupAlgoLast)
            throw rbw::Error(rbw::kInvalidArg, "unknown lookup algorithm");
        const uint32_t k = rbw::lookupHostPipelined(vocOf(voc), static_cast<const uint8_t*>(host_desc), nb_desc,
                                                    host_leaf, static_cast<rbw::LookupAlgo>(algo));
        if (kernels_launched) *kernels_launched = k;
    });
}

int rbw_voc_serialize(const rbw_vocabulary* voc, uint8_t* buf, uint64_t capacity, uint64_t* size)
{
    return guard([&] {
        const auto blob = vocOf(voc).serialize();
        if (size) *size = blob.size();
        if (buf != nullptr) {
            if (capacity < blob.size()) throw rbw::Error(rbw::kInvalidArg, "buffer too small");
            std::memcpy(buf, blob.data(), blob.size());
        }
    });
}

int rbw_voc_deserialize(const uint8_t* blob, uint64_t size, rbw_vocabulary** out)
{
    return guard([&] {
        if (out == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output handle");
        *out = nullptr;
        auto v = rbw::Vocabulary::deserialize(blob, size);
        *out = new rbw_vocabulary{std::move(v)};
    });
}

int rbw_voc_info(const rbw_vocabulary* voc, rbw_desc_attr* attr, uint32_t* branch_factor, uint32_t* nb_levels,
                 uint64_t* nb_nodes)
{
    return guard([&] {
        const auto& v = vocOf(voc);
        if (attr) *attr = rbw_desc_attr{RBW_DATA_UINT8, RBW_DIST_L2, 128};
        if (branch_factor) *branch_factor = v.branch();
        if (nb_levels) *nb_levels = v.levels();
        if (nb_nodes) *nb_nodes = v.nbNodes();
    });
}

int rbw_voc_level_weights(const rbw_vocabulary* voc, uint32_t level, const float** host_weights)
{
    return guard([&] {
        if (host_weights == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output");
        *host_weights = vocOf(voc).levelWeights(level);
    });
}

int rbw_voc_get_tree(const rbw_vocabulary* voc, uint8_t* host_centers, uint32_t* host_masks, float* host_weights)
{
    return guard([&] {
        const auto& v = vocOf(voc);
        if (host_centers) {
            const auto c = v.centersHost();
            std::memcpy(host_centers, c.data(), c.size());
        }
        if (host_masks) std::memcpy(host_masks, v.masks().data(), v.masks().size() * 4);
        if (host_weights) std::memcpy(host_weights, v.weights().data(), v.weights().size() * 4);
    });
}

int rbw_voc_lookup_scratch_bytes(const rbw_vocabulary* voc, uint64_t nb_desc, uint64_t* bytes)
{
    return guard([&] {
        const auto& v = vocOf(voc);
        if (bytes == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output");
        *bytes = rbw::lookupScratchBytes(v.branch(), v.levels(), std::min<uint64_t>(nb_desc, 1ull << 30));
    });
}

int rbw_voc_device_errors(const rbw_vocabulary* voc, uint32_t* code, uint32_t* where)
{
    return guard([&] {
        RBW_CUDA(cudaDeviceSynchronize());
        const rbw::DeviceErrors e = vocOf(voc).takeDeviceErrors();
        if (code) *code = e.code;
        if (where) *where = e.where;
    });
}

void rbw_voc_destroy(rbw_vocabulary* voc) { delete voc; }

int rbw_tuning_set(uint32_t param, uint32_t branch_factor, uint32_t nb_levels, uint32_t bucket, uint32_t value)
{
    return guard([&] {
        if (param >= rbw::kTuneParamCount) throw rbw::Error(rbw::kInvalidArg, "unknown tuning parameter");
        rbw::setTunedValue(static_cast<rbw::TuneParam>(param), branch_factor, nb_levels, bucket, value);
    });
}

int rbw_tuning_get(uint32_t param, uint32_t branch_factor, uint32_t nb_levels, uint64_t n, uint32_t* value)
{
    return guard([&] {
        if (param >= rbw::kTuneParamCount) throw rbw::Error(rbw::kInvalidArg, "unknown tuning parameter");
        if (value == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output");
        *value = rbw::tunedValue(static_cast<rbw::TuneParam>(param), branch_factor, nb_levels, n);
    });
}

int rbw_tuning_clear(void)
{
    return guard([] { rbw::clearTuning(); });
}

void rbw_timing_enable(int32_t on) { rbw::timingEnable(on != 0); }

int rbw_timing_reset(void)
{
    return guard([] { rbw::timingReset(); });
}

int rbw_timing_read(uint32_t kernel, double* total_ms, uint64_t* launches)
{
    return guard([&] {
        if (kernel >= rbw::kTimedCount) throw rbw::Error(rbw::kInvalidArg, "unknown kernel id");
        rbw::timingRead(static_cast<rbw::TimedKernel>(kernel), total_ms, launches);
    });
}

} // extern "C"

namespace rbw {
const Vocabulary& vocabularyOf(const rbw_vocabulary* h) { return vocOf(h); }
int runGuarded(const std::function<void()>& f) { return guard(f); }
} // namespace rbw
