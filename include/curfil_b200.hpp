/*
 * curfil_b200 C++ interface: the reference library's public classes for the training split search and
 * dense prediction path (deeplearningais/curfil, the headers in src/curfil), with the same names, argument
 * meanings and error behaviour (std::runtime_error), implemented over the C-ABI in curfil_b200.h.
 * Header-only; link with libcurfil_b200.so.
 *
 * Every computation of the path runs on the GPU through the C-ABI: integral images, depth filling,
 * feature responses, histograms, scores, candidate generation, training, normalised-histogram
 * packing and prediction. The classes hold host-side data (images, labels, tree nodes) and convert
 * it at the boundary. There is no CPU evaluation path: AccelerationMode CPU_ONLY and
 * GPU_AND_CPU_COMPARE, and predict(..., onGPU = false), throw.
 *
 * Differences from the reference interface (the reference types they replace are named):
 *   - boost::shared_ptr -> std::shared_ptr; cuv::ndarray -> std::vector in the reference layouts.
 *   - Images are built in memory (RGBDImage(width, height), setColor/setDepth); file loading through
 *     Vigra (PNG) is not part of this library.
 *   - PixelInstance::averageRegionDepth/averageRegionColor are not offered on the host; feature
 *     responses are computed on the GPU (ImageFeatureFunction::calculateFeatureResponse).
 *   - RandomTreeImport::readJSON returns the configuration and the tree only (no host name, training
 *     folder or date).
 *   - A device context per GPU is created on first use (the reference's initDevice/selectDevice
 *     globals); curfil::setDefaultDevice chooses the GPU of objects created afterwards.
 */
#ifndef CURFIL_B200_HPP
#define CURFIL_B200_HPP

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <ostream>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "curfil_b200.h"

namespace curfil {

typedef uint8_t LabelType;             // random_tree.h:54
typedef unsigned int WeightType;       // random_tree.h:55
typedef double FeatureResponseType;    // random_tree.h:56
typedef double ScoreType;              // random_tree.h:57

enum HorizontalFlipSetting { NoFlip = 0, Flip = 1, Both = 2 };                 // random_tree.h:58-60
enum SplitBranch { LEFT, RIGHT };                                              // random_tree.h:75-77
enum AccelerationMode { CPU_ONLY, GPU_ONLY, GPU_AND_CPU_COMPARE };             // random_tree.h:79-83
enum FeatureType { DEPTH = 0, COLOR = 1 };                                     // random_tree_image.h:394-396

namespace detail {

// cudaSafeCall / std::runtime_error (utils.h:48): a non-zero status becomes an exception carrying the
// library's message
inline void check(cf_status status) {
    if (status != CF_OK) {
        char msg[4096];
        cf_last_error(msg, sizeof msg);
        throw std::runtime_error(msg);
    }
}

struct DeviceRegistry {
    std::mutex mu;
    std::map<int, cf_context*> contexts;
    int default_device = 0;
    static DeviceRegistry& get() {
        static DeviceRegistry r;
        return r;
    }
};

// The device context of `device` (-1: the default device), created on first use and kept for the
// life of the process (ImageFeatureEvaluation::initDevice, random_tree_image_gpu.cu:1722-1770).
inline cf_context* context(int device = -1) {
    DeviceRegistry& r = DeviceRegistry::get();
    std::lock_guard<std::mutex> lock(r.mu);
    if (device < 0) device = r.default_device;
    auto it = r.contexts.find(device);
    if (it != r.contexts.end()) return it->second;
    cf_context* ctx = nullptr;
    check(cf_context_create(device, &ctx));
    r.contexts[device] = ctx;
    return ctx;
}

inline uint64_t next_image_id() {
    static std::atomic<uint64_t> id{1};
    return id.fetch_add(1);
}

template <class T>
struct Deleter;
template <>
struct Deleter<cf_dataset> {
    void operator()(cf_dataset* p) const { cf_dataset_destroy(p); }
};
template <>
struct Deleter<cf_tree> {
    void operator()(cf_tree* p) const { cf_tree_destroy(p); }
};
template <>
struct Deleter<cf_forest> {
    void operator()(cf_forest* p) const { cf_forest_destroy(p); }
};
template <class T>
using Handle = std::unique_ptr<T, Deleter<T>>;

}  // namespace detail

// Device of the contexts created from now on (the reference's deviceIds[0]).
inline void setDefaultDevice(int device) {
    detail::DeviceRegistry& r = detail::DeviceRegistry::get();
    std::lock_guard<std::mutex> lock(r.mu);
    r.default_device = device;
}

// ---------------------------------------------------------------------------------------------
// Random numbers of the training driver (random_tree.h:1005-1156): a Sampler is an mt19937 seeded
// with its seed and a uniform integer distribution on [lower, upper] (Boost.Random's uniform_int
// bucket method: the engine range 2^32 - 1 split into equal buckets, draws past the last whole bucket
// drawn again); a RandomSource gives every new Sampler the next seed.
// ---------------------------------------------------------------------------------------------
class Sampler {
public:
    Sampler(int seed, int lower, int upper) : seed(seed), lower(lower), upper(upper), rng(static_cast<uint32_t>(seed)) {
        if (upper < lower) throw std::runtime_error("Sampler: upper < lower");
    }
    Sampler(const Sampler& other) : Sampler(other.seed, other.lower, other.upper) {}

    int getNext() {
        const uint32_t range = static_cast<uint32_t>(upper) - static_cast<uint32_t>(lower);
        const uint32_t brange = 0xFFFFFFFFu;
        if (range == 0) return lower;
        if (range == brange) return static_cast<int>(static_cast<uint32_t>(rng()) + static_cast<uint32_t>(lower));
        uint32_t bucket = brange / (range + 1u);
        if (brange % (range + 1u) == range) ++bucket;
        for (;;) {
            const uint32_t r = static_cast<uint32_t>(rng()) / bucket;
            if (r <= range) return static_cast<int>(r + static_cast<uint32_t>(lower));
        }
    }
    int getSeed() const { return seed; }
    int getLower() const { return lower; }
    int getUpper() const { return upper; }

private:
    Sampler& operator=(const Sampler&) = delete;
    int seed, lower, upper;
    std::mt19937 rng;
};

class RandomSource {
public:
    RandomSource(int seed) : seed(seed) {}
    Sampler uniformSampler(int val) { return uniformSampler(0, val - 1); }
    Sampler uniformSampler(int lower, int upper) { return Sampler(seed++, lower, upper); }
    // the seed the next Sampler receives (the training entry points of the C-ABI advance it)
    int& seedCounter() { return seed; }

private:
    int seed;
};

// ---------------------------------------------------------------------------------------------
// TrainingConfiguration (random_tree.h:187-493, random_tree.cpp:114-214)
// ---------------------------------------------------------------------------------------------
class TrainingConfiguration {
public:
    TrainingConfiguration()
        : randomSeed(0), samplesPerImage(0), featureCount(0), minSampleCount(0), maxDepth(0), boxRadius(0),
          regionSize(0), thresholds(0), numThreads(0), maxImages(0), imageCacheSize(0), maxSamplesPerBatch(0),
          accelerationMode(GPU_ONLY), useCIELab(false), useDepthFilling(false), deviceIds(), subsamplingType(),
          ignoredColors(), useDepthImages(false), horizontalFlipping(false) {}

    TrainingConfiguration(int randomSeed, unsigned int samplesPerImage, unsigned int featureCount,
                          unsigned int minSampleCount, int maxDepth, uint16_t boxRadius, uint16_t regionSize,
                          uint16_t thresholds, int numThreads, int maxImages, int imageCacheSize,
                          unsigned int maxSamplesPerBatch, AccelerationMode accelerationMode, bool useCIELab = true,
                          bool useDepthFilling = false, const std::vector<int> deviceIds = std::vector<int>(1, 0),
                          const std::string subsamplingType = "classUniform",
                          const std::vector<std::string>& ignoredColors = std::vector<std::string>(),
                          bool useDepthImages = true, bool horizontalFlipping = false)
        : randomSeed(randomSeed), samplesPerImage(samplesPerImage), featureCount(featureCount),
          minSampleCount(minSampleCount), maxDepth(maxDepth), boxRadius(boxRadius), regionSize(regionSize),
          thresholds(thresholds), numThreads(numThreads), maxImages(maxImages), imageCacheSize(imageCacheSize),
          maxSamplesPerBatch(maxSamplesPerBatch), accelerationMode(accelerationMode), useCIELab(useCIELab),
          useDepthFilling(useDepthFilling), deviceIds(deviceIds), subsamplingType(subsamplingType),
          ignoredColors(ignoredColors), useDepthImages(useDepthImages), horizontalFlipping(horizontalFlipping) {
        for (const std::string& c : ignoredColors)
            if (c.empty()) throw std::runtime_error(std::string("illegal color: '") + c + "'");
        if (maxImages > 0 && maxImages < imageCacheSize) {
            std::ostringstream o;
            o << "illegal configuration: maxImages (" << maxImages << ") must not be lower than imageCacheSize ("
              << imageCacheSize << ")";
            throw std::runtime_error(o.str());
        }
    }

    void setRandomSeed(int s) { randomSeed = s; }
    int getRandomSeed() const { return randomSeed; }
    unsigned int getSamplesPerImage() const { return samplesPerImage; }
    unsigned int getFeatureCount() const { return featureCount; }
    unsigned int getMinSampleCount() const { return minSampleCount; }
    int getMaxDepth() const { return maxDepth; }
    uint16_t getBoxRadius() const { return boxRadius; }
    uint16_t getRegionSize() const { return regionSize; }
    uint16_t getThresholds() const { return thresholds; }
    int getNumThreads() const { return numThreads; }
    int getMaxImages() const { return maxImages; }
    int getImageCacheSize() const { return imageCacheSize; }
    unsigned int getMaxSamplesPerBatch() const { return maxSamplesPerBatch; }
    AccelerationMode getAccelerationMode() const { return accelerationMode; }
    void setAccelerationMode(const AccelerationMode& m) { accelerationMode = m; }
    const std::vector<int>& getDeviceIds() const { return deviceIds; }
    void setDeviceIds(const std::vector<int>& ids) { deviceIds = ids; }
    std::string getSubsamplingType() const { return subsamplingType; }
    bool isUseCIELab() const { return useCIELab; }
    bool isUseDepthFilling() const { return useDepthFilling; }
    bool isUseDepthImages() const { return useDepthImages; }
    bool doHorizontalFlipping() const { return horizontalFlipping; }
    const std::vector<std::string>& getIgnoredColors() const { return ignoredColors; }

    static AccelerationMode parseAccelerationModeString(const std::string& modeString) {
        if (modeString == "cpu") return CPU_ONLY;
        if (modeString == "gpu") return GPU_ONLY;
        if (modeString == "compare") return GPU_AND_CPU_COMPARE;
        throw std::runtime_error(std::string("illegal acceleration mode: ") + modeString);
    }

    std::string getAccelerationModeString() const {
        switch (accelerationMode) {
            case GPU_ONLY: return "gpu";
            case CPU_ONLY: return "cpu";
            case GPU_AND_CPU_COMPARE: return "compare";
        }
        std::ostringstream o;
        o << "unknown acceleration mode: " << static_cast<int>(accelerationMode);
        throw std::runtime_error(o.str());
    }

    // strict also compares the seed, devices, cache size and batch size (random_tree.cpp:160-214)
    bool equals(const TrainingConfiguration& o, bool strict = false) const {
        if (strict && (randomSeed != o.randomSeed || deviceIds != o.deviceIds || imageCacheSize != o.imageCacheSize ||
                       maxSamplesPerBatch != o.maxSamplesPerBatch))
            return false;
        return samplesPerImage == o.samplesPerImage && featureCount == o.featureCount &&
               minSampleCount == o.minSampleCount && maxDepth == o.maxDepth && boxRadius == o.boxRadius &&
               regionSize == o.regionSize && thresholds == o.thresholds && numThreads == o.numThreads &&
               maxImages == o.maxImages && accelerationMode == o.accelerationMode &&
               subsamplingType == o.subsamplingType && ignoredColors == o.ignoredColors && useCIELab == o.useCIELab &&
               useDepthFilling == o.useDepthFilling && useDepthImages == o.useDepthImages &&
               horizontalFlipping == o.horizontalFlipping;
    }
    bool operator==(const TrainingConfiguration& o) const { return equals(o, true); }
    bool operator!=(const TrainingConfiguration& o) const { return !(*this == o); }

    // the C-ABI form (field for field; subsamplingType "classUniform" 0, "pixelUniform" 1)
    cf_train_config toC() const {
        cf_train_config c;
        std::memset(&c, 0, sizeof c);
        c.random_seed = randomSeed;
        c.samples_per_image = samplesPerImage;
        c.feature_count = featureCount;
        c.min_sample_count = minSampleCount;
        c.max_depth = maxDepth;
        c.box_radius = boxRadius;
        c.region_size = regionSize;
        c.thresholds = thresholds;
        c.sampler = 0;
        c.num_threads = numThreads;
        c.max_images = maxImages;
        c.image_cache_size = imageCacheSize;
        c.max_samples_per_batch = maxSamplesPerBatch;
        c.acceleration_mode = static_cast<int32_t>(accelerationMode);
        c.use_cie_lab = useCIELab ? 1 : 0;
        c.use_depth_filling = useDepthFilling ? 1 : 0;
        c.use_depth_images = useDepthImages ? 1 : 0;
        c.horizontal_flipping = horizontalFlipping ? 1 : 0;
        if (subsamplingType == "classUniform")
            c.subsampling_type = 0;
        else if (subsamplingType == "pixelUniform")
            c.subsampling_type = 1;
        else
            throw std::runtime_error("unknown subsampling type: " + subsamplingType);
        return c;
    }

    static TrainingConfiguration fromC(const cf_train_config& c, const std::vector<int>& deviceIds = {0},
                                       const std::vector<std::string>& ignoredColors = {}) {
        return TrainingConfiguration(c.random_seed, c.samples_per_image, c.feature_count, c.min_sample_count,
                                     c.max_depth, c.box_radius, c.region_size, c.thresholds, c.num_threads,
                                     c.max_images, c.image_cache_size, c.max_samples_per_batch,
                                     static_cast<AccelerationMode>(c.acceleration_mode), c.use_cie_lab != 0,
                                     c.use_depth_filling != 0, deviceIds,
                                     c.subsampling_type == 1 ? "pixelUniform" : "classUniform", ignoredColors,
                                     c.use_depth_images != 0, c.horizontal_flipping != 0);
    }

    // the device the configuration names (deviceIds[0], else the default device)
    int device() const { return deviceIds.empty() ? -1 : deviceIds[0]; }

    // fails loudly on the modes this library does not run
    void requireGpu() const {
        if (accelerationMode != GPU_ONLY)
            throw std::runtime_error("acceleration mode '" + getAccelerationModeString() +
                                     "' is not available: this library evaluates on the GPU only");
    }

private:
    int randomSeed;
    unsigned int samplesPerImage;
    unsigned int featureCount;
    unsigned int minSampleCount;
    int maxDepth;
    uint16_t boxRadius;
    uint16_t regionSize;
    uint16_t thresholds;
    int numThreads;
    int maxImages;
    int imageCacheSize;
    unsigned int maxSamplesPerBatch;
    AccelerationMode accelerationMode;
    bool useCIELab;
    bool useDepthFilling;
    std::vector<int> deviceIds;
    std::string subsamplingType;
    std::vector<std::string> ignoredColors;
    bool useDepthImages;
    bool horizontalFlipping;
};

inline std::ostream& operator<<(std::ostream& os, const TrainingConfiguration& c) {
    os << "randomSeed: " << c.getRandomSeed() << ", samplesPerImage: " << c.getSamplesPerImage()
       << ", featureCount: " << c.getFeatureCount() << ", minSampleCount: " << c.getMinSampleCount()
       << ", maxDepth: " << c.getMaxDepth() << ", boxRadius: " << c.getBoxRadius()
       << ", regionSize: " << c.getRegionSize() << ", thresholds: " << c.getThresholds()
       << ", accelerationMode: " << c.getAccelerationModeString() << ", subsamplingType: " << c.getSubsamplingType();
    return os;
}

// ---------------------------------------------------------------------------------------------
// Colours and labels (image.h:51-96, 454-566; image.cpp:40-120, 678-777)
// ---------------------------------------------------------------------------------------------
class RGBColor : public std::vector<uint8_t> {
public:
    RGBColor() : std::vector<uint8_t>(3, 0) {}
    RGBColor(uint8_t r, uint8_t g, uint8_t b) : std::vector<uint8_t>{r, g, b} {}
    // "R,G,B", each 0..255
    RGBColor(const std::string& colorString) : std::vector<uint8_t>(3, 0) {
        std::vector<int> v;
        std::stringstream ss(colorString);
        std::string part;
        while (std::getline(ss, part, ',')) {
            try {
                size_t used = 0;
                const int x = std::stoi(part, &used);
                if (used != part.size()) throw std::invalid_argument("trailing characters");
                v.push_back(x);
            } catch (const std::exception& e) {
                throw std::runtime_error(std::string("illegal color: '") + colorString + "': " + e.what());
            }
        }
        if (v.size() != 3) throw std::runtime_error(std::string("illegal color: '") + colorString + "'");
        for (int x : v)
            if (x < 0 || x > 255) throw std::runtime_error("color value out of range [0-255]: " + colorString);
        (*this)[0] = static_cast<uint8_t>(v[0]);
        (*this)[1] = static_cast<uint8_t>(v[1]);
        (*this)[2] = static_cast<uint8_t>(v[2]);
    }
    std::string toString() const {
        std::ostringstream o;
        o << static_cast<int>((*this)[0]) << "," << static_cast<int>((*this)[1]) << "," << static_cast<int>((*this)[2]);
        return o.str();
    }
};

inline std::ostream& operator<<(std::ostream& os, const RGBColor& c) { return os << c.toString(); }

// Depth in millimetres (image.h:106-188)
class Depth {
public:
    Depth() : value(0) {}
    explicit Depth(const int& value) : value(value) {}
    explicit Depth(const double& metres) : value(static_cast<int>(1000.0 * metres)) {
        if (metres != metres) value = -1;
    }
    bool isValid() const { return value > 0; }
    float getFloatValue() const {
        if (!isValid()) throw std::runtime_error("invalid depth");
        return value / 1000.0f;
    }
    int getIntValue() const { return value; }
    Depth operator-(const Depth& o) const { return Depth(value - o.value); }
    Depth operator+(const Depth& o) const { return Depth(value + o.value); }
    Depth& operator+=(const Depth& o) {
        value += o.value;
        return *this;
    }
    static Depth invalid() { return Depth(-1); }

private:
    int value;
};

class LabelImage {
public:
    LabelImage(int width, int height)
        : width(width), height(height), image(static_cast<size_t>(std::max(0, width)) * std::max(0, height), 0) {
        if (width < 0 || height < 0) throw std::runtime_error("LabelImage: negative size");
    }
    int getWidth() const { return width; }
    int getHeight() const { return height; }
    bool isInImage(int x, int y) const { return x >= 0 && x < width && y >= 0 && y < height; }
    void setLabel(int x, int y, const LabelType label) { image[static_cast<size_t>(y) * width + x] = label; }
    LabelType getLabel(int x, int y) const { return image[static_cast<size_t>(y) * width + x]; }
    size_t getSizeInMemory() const { return image.size() * sizeof(LabelType); }
    const LabelType* data() const { return image.data(); }
    LabelType* data() { return image.data(); }

    // the label of a colour: colours get ids in the order they are first seen (image.cpp:678-687)
    static LabelType encodeColor(RGBColor color) {
        Registry& r = registry();
        std::lock_guard<std::mutex> lock(r.mu);
        auto it = r.colors.find(color);
        if (it != r.colors.end()) return it->second;
        const LabelType id = static_cast<LabelType>(r.colors.size());
        r.colors[color] = id;
        return id;
    }
    static RGBColor decodeLabel(const LabelType& v) {
        Registry& r = registry();
        std::lock_guard<std::mutex> lock(r.mu);
        for (auto& kv : r.colors)
            if (kv.second == v) return kv.first;
        std::ostringstream o;
        o << "color for label " << static_cast<int>(v) << " not found";
        throw std::runtime_error(o.str());
    }
    // LabelImage::resizeImage (image.cpp:763-777): the image in the top-left corner, paddingLabel elsewhere
    void resizeImage(int newWidth, int newHeight, LabelType paddingLabel) {
        std::vector<LabelType> out(static_cast<size_t>(newWidth) * newHeight, paddingLabel);
        for (int y = 0; y < std::min(height, newHeight); y++)
            for (int x = 0; x < std::min(width, newWidth); x++)
                out[static_cast<size_t>(y) * newWidth + x] = image[static_cast<size_t>(y) * width + x];
        image.swap(out);
        width = newWidth;
        height = newHeight;
    }

private:
    struct Registry {
        std::mutex mu;
        std::map<RGBColor, LabelType> colors;
    };
    static Registry& registry() {
        static Registry r;
        return r;
    }
    int width, height;
    std::vector<LabelType> image;
};

// getPaddingLabel (image.cpp:858-867): the first ignored colour's label, else black's
inline LabelType getPaddingLabel(const std::vector<std::string>& ignoredColors) {
    return LabelImage::encodeColor(ignoredColors.empty() ? RGBColor(0, 0, 0) : RGBColor(ignoredColors[0]));
}

// ---------------------------------------------------------------------------------------------
// RGBDImage (image.h:201-446): colour float [3][H][W], depth int [2][H][W] = {mm (0 invalid), valid}
// ---------------------------------------------------------------------------------------------
class RGBDImage {
public:
    static const int COLOR_CHANNELS = 3;
    static const int DEPTH_CHANNELS = 2;

    RGBDImage(int width, int height) : width(width), height(height), id(detail::next_image_id()) {
        if (width < 0 || height < 0) throw std::runtime_error("RGBDImage: negative size");
        reset();
    }
    RGBDImage(const RGBDImage& o)
        : width(o.width), height(o.height), colorImage(o.colorImage), depthImage(o.depthImage), inCIELab(o.inCIELab),
          integratedColor(o.integratedColor), integratedDepth(o.integratedDepth), id(detail::next_image_id()) {}

    // convenience: a frame from raw interleaved uint8 RGB [H][W][3] and depth mm [H][W] (0 = missing)
    static RGBDImage fromRaw(int width, int height, const uint8_t* rgb, const uint16_t* depthMm) {
        RGBDImage im(width, height);
        const size_t plane = static_cast<size_t>(width) * height;
        for (size_t p = 0; p < plane; p++) {
            for (int c = 0; c < COLOR_CHANNELS; c++) im.colorImage[c * plane + p] = rgb[3 * p + c];
            im.depthImage[p] = depthMm[p];
            im.depthImage[plane + p] = depthMm[p] > 0 ? 1 : 0;
        }
        return im;
    }

    int getWidth() const { return width; }
    int getHeight() const { return height; }
    size_t getSizeInMemory() const { return colorImage.size() * sizeof(float) + depthImage.size() * sizeof(int); }
    bool hasIntegratedDepth() const { return integratedDepth; }
    bool hasIntegratedColor() const { return integratedColor; }
    bool inImage(int x, int y) const { return x >= 0 && x < width && y >= 0 && y < height; }

    void reset() {
        colorImage.assign(static_cast<size_t>(COLOR_CHANNELS) * width * height, 0.0f);
        depthImage.assign(static_cast<size_t>(DEPTH_CHANNELS) * width * height, 0);
        integratedColor = integratedDepth = inCIELab = false;
        touch();
    }
    // invalid depth is stored as 0, which the integral needs (image.h:363-371)
    void setDepth(int x, int y, const Depth& depth) {
        const size_t p = static_cast<size_t>(y) * width + x;
        depthImage[p] = depth.isValid() ? depth.getIntValue() : 0;
        depthImage[static_cast<size_t>(width) * height + p] = depth.isValid() ? 1 : 0;
        touch();
    }
    Depth getDepth(int x, int y) const { return Depth(depthImage[static_cast<size_t>(y) * width + x]); }
    int getDepthValid(int x, int y) const {
        return depthImage[static_cast<size_t>(width) * height + static_cast<size_t>(y) * width + x];
    }
    void setColor(int x, int y, unsigned int channel, float color) {
        colorImage[static_cast<size_t>(channel) * width * height + static_cast<size_t>(y) * width + x] = color;
        touch();
    }
    float getColor(int x, int y, unsigned int channel) const {
        return colorImage[static_cast<size_t>(channel) * width * height + static_cast<size_t>(y) * width + x];
    }
    const std::vector<float>& getColorImage() const { return colorImage; }
    const std::vector<int>& getDepthImage() const { return depthImage; }

    // RGBDImage::calculateIntegral (image.cpp:531-556), on the GPU
    void calculateIntegral() {
        if (integratedColor || integratedDepth) throw std::runtime_error("image already integrated");
        if (width == 0 || height == 0) {
            integratedColor = integratedDepth = true;
            return;
        }
        detail::check(cf_integrate_planes(detail::context(), 1, width, height, colorImage.data(), depthImage.data(),
                                          colorImage.data(), depthImage.data(), 0));
        integratedColor = integratedDepth = true;
        touch();
    }

    // RGBDImage::fillDepth (image.cpp:279-377), on the GPU; before integration
    void fillDepth() {
        if (integratedDepth) throw std::runtime_error("fillDepth: image already integrated");
        const size_t plane = static_cast<size_t>(width) * height;
        std::vector<uint16_t> d(plane);
        for (size_t p = 0; p < plane; p++) {
            if (depthImage[p] < 0 || depthImage[p] > 65535) throw std::runtime_error("fillDepth: depth out of range");
            d[p] = static_cast<uint16_t>(depthImage[p]);
        }
        if (plane) detail::check(cf_fill_depth(detail::context(), 1, width, height, d.data(), 0));
        for (size_t p = 0; p < plane; p++) {
            depthImage[p] = d[p];
            depthImage[plane + p] = d[p] > 0 ? 1 : 0;
        }
        touch();
    }

    // RGBDImage::loadDummyDepthValues (image.cpp:379-394): 1 m everywhere (useDepthImages = false)
    void loadDummyDepthValues() {
        const size_t plane = static_cast<size_t>(width) * height;
        for (size_t p = 0; p < plane; p++) {
            depthImage[p] = 1000;
            depthImage[plane + p] = 1;
        }
        touch();
    }

    // RGBDImage::resizeImage (image.cpp:450-475): colour NaN and depth 0 outside the original frame
    void resizeImage(int newWidth, int newHeight) {
        const size_t np = static_cast<size_t>(newWidth) * newHeight, op = static_cast<size_t>(width) * height;
        std::vector<float> ci(COLOR_CHANNELS * np, std::numeric_limits<float>::quiet_NaN());
        std::vector<int> di(DEPTH_CHANNELS * np, 0);
        for (int y = 0; y < std::min(height, newHeight); y++)
            for (int x = 0; x < std::min(width, newWidth); x++) {
                const size_t s = static_cast<size_t>(y) * width + x, d = static_cast<size_t>(y) * newWidth + x;
                for (int c = 0; c < COLOR_CHANNELS; c++) ci[c * np + d] = colorImage[c * op + s];
                for (int c = 0; c < DEPTH_CHANNELS; c++) di[c * np + d] = depthImage[c * op + s];
            }
        colorImage.swap(ci);
        depthImage.swap(di);
        width = newWidth;
        height = newHeight;
        touch();
    }

    // identity of the current contents (changes with every modification); keys the device image cache
    std::pair<uint64_t, uint64_t> cacheKey() const { return std::make_pair(id, version); }

private:
    void touch() { version++; }
    int width, height;
    std::vector<float> colorImage;
    std::vector<int> depthImage;
    bool inCIELab = false, integratedColor = false, integratedDepth = false;
    uint64_t id;
    uint64_t version = 0;
};

class LabeledRGBDImage {
public:
    std::shared_ptr<RGBDImage> rgbdImage;
    std::shared_ptr<LabelImage> labelImage;

    LabeledRGBDImage() {}
    LabeledRGBDImage(const std::shared_ptr<RGBDImage>& rgbdImage, const std::shared_ptr<LabelImage>& labelImage)
        : rgbdImage(rgbdImage), labelImage(labelImage) {
        if (rgbdImage->getWidth() != labelImage->getWidth() || rgbdImage->getHeight() != labelImage->getHeight()) {
            std::ostringstream o;
            o << "RGB-D image and label image have different sizes: " << rgbdImage->getWidth() << "x"
              << rgbdImage->getHeight() << " and " << labelImage->getWidth() << "x" << labelImage->getHeight();
            throw std::runtime_error(o.str());
        }
    }
    size_t getSizeInMemory() const { return rgbdImage->getSizeInMemory() + labelImage->getSizeInMemory(); }
    const RGBDImage& getRGBDImage() const { return *rgbdImage; }
    const LabelImage& getLabelImage() const { return *labelImage; }
    int getWidth() const { return rgbdImage->getWidth(); }
    int getHeight() const { return rgbdImage->getHeight(); }
    void resizeImage(int newWidth, int newHeight, LabelType paddingLabel) const {
        rgbdImage->resizeImage(newWidth, newHeight);
        labelImage->resizeImage(newWidth, newHeight, paddingLabel);
    }
    void calculateIntegral() const { rgbdImage->calculateIntegral(); }
};

// ---------------------------------------------------------------------------------------------
// XY, PixelInstance (random_tree_image.h:40-390)
// ---------------------------------------------------------------------------------------------
class XY {
public:
    XY() : x(0), y(0) {}
    XY(int x, int y) : x(x), y(y) {}
    // XY::normalize (random_tree_image.h:82-87): int / float, truncated
    XY normalize(const Depth& depth) const {
        const float d = depth.getFloatValue();
        return XY(static_cast<int>(x / d), static_cast<int>(y / d));
    }
    bool operator==(const XY& o) const { return x == o.x && y == o.y; }
    bool operator!=(const XY& o) const { return !(*this == o); }
    int getX() const { return x; }
    int getY() const { return y; }

private:
    int x, y;
};
typedef XY Region;
typedef XY Offset;
typedef XY Point;

class PixelInstance {
public:
    // the pixel's depth recovered from the integrated depth image (random_tree_image.h:140-165)
    PixelInstance(const RGBDImage* image, const LabelType& label, uint16_t x, uint16_t y,
                  HorizontalFlipSetting setting = NoFlip)
        : image(image), label(label), point(x, y), depth(Depth::invalid()), horFlipSetting(setting) {
        if (!image) throw std::runtime_error("PixelInstance: image is NULL");
        if (!image->inImage(x, y)) throw std::runtime_error("PixelInstance: pixel outside the image");
        if (!image->hasIntegratedDepth()) throw std::runtime_error("image is not integrated");
        const int aboveValid = (y > 0) ? image->getDepthValid(x, y - 1) : 0;
        const int leftValid = (x > 0) ? image->getDepthValid(x - 1, y) : 0;
        const int aboveLeftValid = (x > 0 && y > 0) ? image->getDepthValid(x - 1, y - 1) : 0;
        const int valid = image->getDepthValid(x, y) - (leftValid + aboveValid - aboveLeftValid);
        if (valid == 1) {
            const int above = (y > 0) ? image->getDepth(x, y - 1).getIntValue() : 0;
            const int left = (x > 0) ? image->getDepth(x - 1, y).getIntValue() : 0;
            const int aboveLeft = (x > 0 && y > 0) ? image->getDepth(x - 1, y - 1).getIntValue() : 0;
            const uint32_t mm = static_cast<uint32_t>(image->getDepth(x, y).getIntValue()) -
                                (static_cast<uint32_t>(left) + static_cast<uint32_t>(above) -
                                 static_cast<uint32_t>(aboveLeft));
            depth = Depth(static_cast<int>(mm));
        }
    }
    PixelInstance(const RGBDImage* image, const LabelType& label, const Depth& depth, uint16_t x, uint16_t y,
                  HorizontalFlipSetting setting = NoFlip)
        : image(image), label(label), point(x, y), depth(depth), horFlipSetting(setting) {}

    const RGBDImage* getRGBDImage() const { return image; }
    int width() const { return image->getWidth(); }
    int height() const { return image->getHeight(); }
    uint16_t getX() const { return static_cast<uint16_t>(point.getX()); }
    uint16_t getY() const { return static_cast<uint16_t>(point.getY()); }
    LabelType getLabel() const { return label; }
    const Depth getDepth() const { return depth; }
    WeightType getWeight() const { return 1; }
    HorizontalFlipSetting getHorFlipSetting() const { return horFlipSetting; }
    void setHorFlipSetting(HorizontalFlipSetting s) { horFlipSetting = s; }
    float getColor(const Point& pos, uint8_t channel) const { return image->getColor(pos.getX(), pos.getY(), channel); }
    Depth getDepth(const Point& pos) const { return image->getDepth(pos.getX(), pos.getY()); }
    int getDepthValid(const Point& pos) const { return image->getDepthValid(pos.getX(), pos.getY()); }
    bool inImage(int x, int y) const { return image->inImage(x, y); }
    bool inImage(const Point& pos) const { return inImage(pos.getX(), pos.getY()); }

    // the C-ABI sample for an image at `imageIndex` of a device dataset
    cf_sample toSample(uint32_t imageIndex) const {
        cf_sample s;
        std::memset(&s, 0, sizeof s);
        s.x = getX();
        s.y = getY();
        s.image = imageIndex;
        s.depth = depth.isValid() ? depth.getFloatValue() : 0.0f;
        s.label = label;
        s.flip = static_cast<uint8_t>(horFlipSetting);
        return s;
    }

private:
    const RGBDImage* image;
    LabelType label;
    Point point;
    Depth depth;
    HorizontalFlipSetting horFlipSetting;
};

namespace detail {

// Integrated images on the device (ImageCache, random_tree_image_gpu.cu:727-908): the distinct
// images of a set of instances uploaded into one dataset, in first-seen order.
class DeviceImages {
public:
    explicit DeviceImages(int device = -1) : device(device) {}

    template <class Instances, class Get>
    std::vector<cf_sample> upload(const Instances& instances, Get get) {
        std::map<std::pair<uint64_t, uint64_t>, uint32_t> index;
        std::vector<const RGBDImage*> images;
        std::vector<cf_sample> samples;
        samples.reserve(instances.size());
        for (const auto& item : instances) {
            const PixelInstance& inst = get(item);
            const RGBDImage* im = inst.getRGBDImage();
            auto key = im->cacheKey();
            auto it = index.find(key);
            uint32_t k;
            if (it == index.end()) {
                k = static_cast<uint32_t>(images.size());
                index[key] = k;
                images.push_back(im);
            } else {
                k = it->second;
            }
            samples.push_back(inst.toSample(k));
        }
        if (images.empty()) throw std::runtime_error("no samples");
        const int W = images[0]->getWidth(), H = images[0]->getHeight();
        for (const RGBDImage* im : images) {
            if (im->getWidth() != W || im->getHeight() != H)
                throw std::runtime_error("all images must have the same size (resize them to the largest frame)");
            if (!im->hasIntegratedColor() || !im->hasIntegratedDepth())
                throw std::runtime_error("image is not integrated");
        }
        upload_images(images);
        return samples;
    }

    void upload_images(const std::vector<const RGBDImage*>& images) {
        const int n = static_cast<int>(images.size());
        const int W = images[0]->getWidth(), H = images[0]->getHeight();
        cf_dataset* raw = nullptr;
        check(cf_dataset_create(context(device), n, W, H, &raw));
        ds.reset(raw);
        for (int i = 0; i < n; i++)
            check(cf_dataset_upload_integral(raw, i, 1, images[i]->getColorImage().data(),
                                             images[i]->getDepthImage().data()));
    }

    cf_dataset* get() const { return ds.get(); }

private:
    int device;
    Handle<cf_dataset> ds;
};

inline const PixelInstance& as_instance(const PixelInstance& p) { return p; }
inline const PixelInstance& as_instance(const PixelInstance* p) { return *p; }

}  // namespace detail

// ---------------------------------------------------------------------------------------------
// ImageFeatureFunction (random_tree_image.h:404-625)
// ---------------------------------------------------------------------------------------------
class ImageFeatureFunction {
public:
    ImageFeatureFunction(FeatureType featureType, const Offset& offset1, const Region& region1, const uint8_t channel1,
                         const Offset& offset2, const Region& region2, const uint8_t channel2)
        : featureType(featureType), offset1(offset1), region1(region1), channel1(channel1), offset2(offset2),
          region2(region2), channel2(channel2) {
        if (offset1 == offset2) throw std::runtime_error("illegal feature: offset1 equals offset2");
    }
    ImageFeatureFunction() : featureType(DEPTH), channel1(0), channel2(0) {}

    // getSortKey (random_tree_image.h:444-452)
    int getSortKey() const {
        int32_t key = 0;
        key |= static_cast<uint8_t>(getType() & 0x03) << 30;
        key |= static_cast<uint8_t>(getChannel1() & 0x0F) << 26;
        key |= static_cast<uint8_t>(getChannel2() & 0x0F) << 22;
        key |= static_cast<uint8_t>((getOffset1().getY() + 127) & 0xFF) << 14;
        key |= static_cast<uint8_t>((getOffset1().getX() + 127) & 0xFF) << 6;
        return key;
    }
    FeatureType getType() const { return featureType; }
    std::string getTypeString() const {
        switch (featureType) {
            case COLOR: return "color";
            case DEPTH: return "depth";
        }
        throw std::runtime_error("unknown feature");
    }
    bool isValid() const { return offset1 != offset2; }
    const Offset& getOffset1() const { return offset1; }
    const Region& getRegion1() const { return region1; }
    uint8_t getChannel1() const { return channel1; }
    const Offset& getOffset2() const { return offset2; }
    const Region& getRegion2() const { return region2; }
    uint8_t getChannel2() const { return channel2; }
    bool operator==(const ImageFeatureFunction& o) const {
        return featureType == o.featureType && offset1 == o.offset1 && region1 == o.region1 &&
               channel1 == o.channel1 && offset2 == o.offset2 && region2 == o.region2 && channel2 == o.channel2;
    }
    bool operator!=(const ImageFeatureFunction& o) const { return !(*this == o); }

    // the 11 table parameters (random_tree_image.h:686-759 row order)
    void toColumn(int8_t out[11]) const {
        out[0] = static_cast<int8_t>(featureType);
        out[1] = static_cast<int8_t>(offset1.getX());
        out[2] = static_cast<int8_t>(offset1.getY());
        out[3] = static_cast<int8_t>(offset2.getX());
        out[4] = static_cast<int8_t>(offset2.getY());
        out[5] = static_cast<int8_t>(region1.getX());
        out[6] = static_cast<int8_t>(region1.getY());
        out[7] = static_cast<int8_t>(region2.getX());
        out[8] = static_cast<int8_t>(region2.getY());
        out[9] = static_cast<int8_t>(channel1);
        out[10] = static_cast<int8_t>(channel2);
    }
    static ImageFeatureFunction fromColumn(const int8_t f[11]) {
        ImageFeatureFunction r;
        r.featureType = static_cast<FeatureType>(f[0]);
        r.offset1 = Offset(f[1], f[2]);
        r.offset2 = Offset(f[3], f[4]);
        r.region1 = Region(f[5], f[6]);
        r.region2 = Region(f[7], f[8]);
        r.channel1 = static_cast<uint8_t>(f[9]);
        r.channel2 = static_cast<uint8_t>(f[10]);
        return r;
    }

    // calculateFeatureResponse (random_tree_image.h:485-497), evaluated on the GPU
    FeatureResponseType calculateFeatureResponse(const PixelInstance& instance, bool flipRegion = false) const {
        PixelInstance inst = instance;
        inst.setHorFlipSetting(flipRegion ? Flip : NoFlip);
        std::vector<PixelInstance> one(1, inst);
        return calculateFeatureResponses(one)[0];
    }

    // responses of many instances at once (one launch); the flip of each instance applies (Both: NoFlip)
    template <class Instances>
    std::vector<FeatureResponseType> calculateFeatureResponses(const Instances& instances) const {
        detail::DeviceImages images;
        std::vector<cf_sample> samples =
            images.upload(instances, [](const typename Instances::value_type& v) -> const PixelInstance& {
                return detail::as_instance(v);
            });
        for (cf_sample& s : samples)
            if (s.flip == Both) s.flip = NoFlip;
        int8_t column[11];
        toColumn(column);
        std::vector<FeatureResponseType> out(samples.size());
        detail::check(cf_feature_responses(images.get(), static_cast<int>(samples.size()), samples.data(), 1, column,
                                           out.data()));
        return out;
    }

private:
    FeatureType featureType;
    Offset offset1;
    Region region1;
    uint8_t channel1;
    Offset offset2;
    Region region2;
    uint8_t channel2;
};

inline std::ostream& operator<<(std::ostream& os, const ImageFeatureFunction& f) {
    os << f.getTypeString() << ", offset1: " << f.getOffset1().getX() << "," << f.getOffset1().getY()
       << ", region1: " << f.getRegion1().getX() << "," << f.getRegion1().getY()
       << ", offset2: " << f.getOffset2().getX() << "," << f.getOffset2().getY()
       << ", region2: " << f.getRegion2().getX() << "," << f.getRegion2().getY();
    if (f.getType() == COLOR) os << ", channels: " << int(f.getChannel1()) << "," << int(f.getChannel2());
    return os;
}

// ---------------------------------------------------------------------------------------------
// ImageFeaturesAndThresholds (random_tree_image.h:635-912), host memory: features int8 [11][F],
// thresholds float [T][F]
// ---------------------------------------------------------------------------------------------
class ImageFeaturesAndThresholds {
public:
    ImageFeaturesAndThresholds(size_t numFeatures, size_t numThresholds)
        : F(numFeatures), T(numThresholds), m_features(11 * numFeatures, 0), m_thresholds(numThresholds * numFeatures, 0.0f) {}

    size_t numFeatures() const { return F; }
    size_t numThresholds() const { return T; }
    const int8_t* features() const { return m_features.data(); }
    int8_t* features() { return m_features.data(); }
    const float* thresholds() const { return m_thresholds.data(); }
    float* thresholds() { return m_thresholds.data(); }
    const int8_t* types() const { return row(0); }
    const int8_t* offset1X() const { return row(1); }
    const int8_t* offset1Y() const { return row(2); }
    const int8_t* offset2X() const { return row(3); }
    const int8_t* offset2Y() const { return row(4); }
    const int8_t* region1X() const { return row(5); }
    const int8_t* region1Y() const { return row(6); }
    const int8_t* region2X() const { return row(7); }
    const int8_t* region2Y() const { return row(8); }
    const int8_t* channel1() const { return row(9); }
    const int8_t* channel2() const { return row(10); }

    double getThreshold(size_t threshNr, size_t featNr) const { return m_thresholds[threshNr * F + featNr]; }
    void setThreshold(size_t threshNr, size_t featNr, float v) { m_thresholds[threshNr * F + featNr] = v; }
    void setFeatureFunction(size_t feat, const ImageFeatureFunction& feature) {
        int8_t c[11];
        feature.toColumn(c);
        for (int r = 0; r < 11; r++) m_features[r * F + feat] = c[r];
    }
    ImageFeatureFunction getFeatureFunction(size_t feat) const {
        int8_t c[11];
        for (int r = 0; r < 11; r++) c[r] = m_features[r * F + feat];
        return ImageFeatureFunction::fromColumn(c);
    }

private:
    const int8_t* row(int r) const { return m_features.data() + r * F; }
    size_t F, T;
    std::vector<int8_t> m_features;
    std::vector<float> m_thresholds;
};

// ---------------------------------------------------------------------------------------------
// SplitFunction and RandomTree (random_tree.h:100-180, 499-1003)
// ---------------------------------------------------------------------------------------------
template <class Instance, class FeatureFunction>
class SplitFunction {
public:
    SplitFunction(size_t featureId, const FeatureFunction& feature, float threshold, ScoreType score)
        : featureId(featureId), feature(feature), threshold(threshold), score(score) {}
    SplitFunction()
        : featureId(0), feature(), threshold(std::numeric_limits<float>::quiet_NaN()),
          score(std::numeric_limits<float>::quiet_NaN()) {}

    // SplitFunction::split (random_tree.h:122-144): response <= threshold goes left; responses on GPU
    SplitBranch split(const Instance& instance, bool& flippedSameSplit) const {
        flippedSameSplit = true;
        const HorizontalFlipSetting s = instance.getHorFlipSetting();
        if (s == Both) {
            const bool a = feature.calculateFeatureResponse(instance) <= getThreshold();
            const bool b = feature.calculateFeatureResponse(instance, true) <= getThreshold();
            if (a != b) flippedSameSplit = false;
            return a ? LEFT : RIGHT;
        }
        const bool v = feature.calculateFeatureResponse(instance, s == Flip) <= getThreshold();
        return v ? LEFT : RIGHT;
    }
    const FeatureFunction& getFeature() const { return feature; }
    float getThreshold() const { return threshold; }
    ScoreType getScore() const { return score; }
    size_t getFeatureId() const { return featureId; }

private:
    size_t featureId;
    FeatureFunction feature;
    float threshold;
    ScoreType score;
};

template <class Instance, class FeatureFunction>
class RandomTree {
public:
    typedef std::shared_ptr<RandomTree> Ptr;

    RandomTree(size_t nodeId, int level, const std::vector<WeightType>& histogram, size_t treeId = 0,
               const RandomTree* parent = nullptr)
        : nodeId(nodeId), treeId(treeId), level(level), parent(parent), histogram(histogram) {}

    bool isRoot() const { return parent == nullptr; }
    const RandomTree* getRoot() const { return parent ? parent->getRoot() : this; }
    bool isLeaf() const { return !left; }
    std::shared_ptr<const RandomTree> getLeft() const { return left; }
    std::shared_ptr<const RandomTree> getRight() const { return right; }
    const SplitFunction<Instance, FeatureFunction>& getSplit() const { return split; }
    int getLevel() const { return level; }
    size_t getNodeId() const { return nodeId; }
    size_t getTreeId() const { return treeId; }
    size_t getNumClasses() const { return histogram.size(); }
    size_t getNumTrainSamples() const { return numTrainSamples; }
    const std::vector<WeightType>& getHistogram() const { return histogram; }
    const std::vector<double>& getNormalizedHistogram() const { return normalizedHistogram; }

    bool hasPureHistogram() const {
        int nonZero = 0;
        for (WeightType h : histogram) nonZero += h > 0;
        return nonZero <= 1;
    }
    size_t countNodes() const { return 1 + (isLeaf() ? 0 : left->countNodes() + right->countNodes()); }
    size_t countLeafNodes() const { return isLeaf() ? 1 : left->countLeafNodes() + right->countLeafNodes(); }
    size_t getTreeDepth() const {
        return isLeaf() ? 1 : 1 + std::max(left->getTreeDepth(), right->getTreeDepth());
    }
    void collectLeafNodes(std::vector<size_t>& leafSet) const {
        if (isLeaf())
            leafSet.push_back(nodeId);
        else {
            left->collectLeafNodes(leafSet);
            right->collectLeafNodes(leafSet);
        }
    }
    LabelType getDominantClass() const {
        const std::vector<double>& h = normalizedHistogram.empty() ? toDouble() : normalizedHistogram;
        LabelType best = 0;
        for (size_t c = 1; c < h.size(); c++)
            if (h[c] > h[best]) best = static_cast<LabelType>(c);
        return best;
    }

    // detail::normalizeHistogram of every node (random_tree.h:822-847, random_tree.cpp:54-104)
    void normalizeHistograms(const std::vector<WeightType>& priorDistribution, const double histogramBias,
                             const bool useLabelsPrior) {
        normalizedHistogram.assign(histogram.size(), 0.0);
        detail::check(cf_normalize_histogram(static_cast<int>(histogram.size()), histogram.data(),
                                             priorDistribution.data(), histogramBias, useLabelsPrior ? 1 : 0,
                                             normalizedHistogram.data()));
        if (!isLeaf()) {
            left->normalizeHistograms(priorDistribution, histogramBias, useLabelsPrior);
            right->normalizeHistograms(priorDistribution, histogramBias, useLabelsPrior);
        }
    }

    // traverseToLeaf / classifySoft / classify (random_tree.h:613-622, 989-1002); responses on GPU
    const RandomTree* traverseToLeaf(const Instance& instance) const {
        const RandomTree* node = this;
        while (!node->isLeaf()) {
            bool same = true;
            node = node->split.split(instance, same) == LEFT ? node->left.get() : node->right.get();
        }
        return node;
    }
    const std::vector<double>& classifySoft(const Instance& instance) const {
        return traverseToLeaf(instance)->getNormalizedHistogram();
    }
    LabelType classify(const Instance& instance) const { return traverseToLeaf(instance)->getDominantClass(); }

    // building (RandomTree::addChildren, random_tree.h:763-790)
    void addChildren(const SplitFunction<Instance, FeatureFunction>& s, Ptr leftChild, Ptr rightChild) {
        split = s;
        left = leftChild;
        right = rightChild;
    }
    void setNumTrainSamples(size_t n) { numTrainSamples = n; }

private:
    std::vector<double> toDouble() const { return std::vector<double>(histogram.begin(), histogram.end()); }
    size_t nodeId, treeId;
    int level;
    const RandomTree* parent;
    std::vector<WeightType> histogram;
    std::vector<double> normalizedHistogram;
    size_t numTrainSamples = 0;
    SplitFunction<Instance, FeatureFunction> split;
    Ptr left, right;
};

typedef RandomTree<PixelInstance, ImageFeatureFunction> ImageTree;

namespace detail {

// The breadth-first node arrays of a trained cf_tree as RandomTree nodes (node id = treeId + index).
inline std::shared_ptr<ImageTree> build_tree(cf_tree* tree) {
    int n = 0, C = 0, depth = 0, treeId = 0;
    check(cf_tree_info(tree, &n, &C, &depth, &treeId));
    std::vector<int32_t> level(n), left(n), featureId(n);
    std::vector<int8_t> feature(static_cast<size_t>(n) * 11);
    std::vector<float> threshold(n);
    std::vector<double> score(n);
    std::vector<uint32_t> hist(static_cast<size_t>(n) * C), samples(n);
    check(cf_tree_export(tree, level.data(), left.data(), feature.data(), threshold.data(), score.data(),
                         featureId.data(), hist.data(), samples.data()));
    std::vector<std::shared_ptr<ImageTree>> nodes(n);
    std::vector<const ImageTree*> parents(n, nullptr);
    for (int i = 0; i < n; i++) {
        std::vector<WeightType> h(hist.begin() + static_cast<size_t>(i) * C, hist.begin() + static_cast<size_t>(i + 1) * C);
        nodes[i] = std::make_shared<ImageTree>(static_cast<size_t>(treeId + i), level[i], h, treeId, parents[i]);
        nodes[i]->setNumTrainSamples(samples[i]);
        if (left[i] >= 0) {
            if (left[i] <= i || left[i] + 1 >= n) throw std::runtime_error("corrupt tree: child index");
            parents[left[i]] = parents[left[i] + 1] = nodes[i].get();
        }
    }
    for (int i = n - 1; i >= 0; i--) {
        if (left[i] < 0) continue;
        SplitFunction<PixelInstance, ImageFeatureFunction> s(
            static_cast<size_t>(featureId[i]), ImageFeatureFunction::fromColumn(&feature[static_cast<size_t>(i) * 11]),
            threshold[i], score[i]);
        nodes[i]->addChildren(s, nodes[left[i]], nodes[left[i] + 1]);
    }
    return nodes.empty() ? nullptr : nodes[0];
}

inline std::vector<uint8_t> ignored_mask(const TrainingConfiguration& c, size_t numLabels) {
    std::vector<uint8_t> mask(std::max<size_t>(numLabels, 1), 0);
    for (const std::string& color : c.getIgnoredColors()) {
        const LabelType l = LabelImage::encodeColor(RGBColor(color));
        if (l < mask.size()) mask[l] = 1;
    }
    return mask;
}

}  // namespace detail

// ---------------------------------------------------------------------------------------------
// ImageFeatureEvaluation (random_tree_image.h:988-1096; random_tree_image.cpp:239-502;
// random_tree_image_gpu.cu:1853-2182)
// ---------------------------------------------------------------------------------------------
class ImageFeatureEvaluation {
public:
    ImageFeatureEvaluation(const size_t treeId, const TrainingConfiguration& configuration)
        : treeId(treeId), configuration(configuration) {
        if (configuration.getBoxRadius() == 0 || configuration.getRegionSize() == 0)
            throw std::runtime_error("boxRadius and regionSize must be > 0");
        configuration.requireGpu();
        detail::context(configuration.device());
    }

    // generateRandomFeatures (GPU form, random_tree_image_gpu.cu:1896-1956 + sortFeatures): thresholds
    // are the responses of random samples of `samples`; the table is sorted by getSortKey when `sort`
    ImageFeaturesAndThresholds generateRandomFeatures(const std::vector<const PixelInstance*>& samples, int seed,
                                                      const bool sort = true) const {
        if (!sort) throw std::runtime_error("generateRandomFeatures: the GPU candidate table is always sorted");
        detail::DeviceImages images(configuration.device());
        std::vector<cf_sample> s = images.upload(samples, [](const PixelInstance* p) -> const PixelInstance& {
            return *p;
        });
        ImageFeaturesAndThresholds ft(configuration.getFeatureCount(), configuration.getThresholds());
        detail::check(cf_generate_features(images.get(), static_cast<int>(s.size()), s.data(),
                                           static_cast<uint32_t>(seed), static_cast<int>(ft.numFeatures()),
                                           static_cast<int>(ft.numThresholds()), configuration.getBoxRadius(),
                                           configuration.getRegionSize(), configuration.isUseDepthImages() ? 1 : 0,
                                           ft.features(), ft.thresholds()));
        return ft;
    }

    // calculateFeatureResponsesAndHistograms (random_tree_image_gpu.cu:1958-2135): counters uint32
    // [F][T][C][2] over all batches; featureResponsesHost (optional) receives the responses [F][N]
    std::vector<WeightType> calculateFeatureResponsesAndHistograms(
        size_t numClasses, const std::vector<std::vector<const PixelInstance*>>& batches,
        const ImageFeaturesAndThresholds& ft, std::vector<FeatureResponseType>* featureResponsesHost = nullptr) const {
        std::vector<const PixelInstance*> all;
        for (const auto& b : batches) all.insert(all.end(), b.begin(), b.end());
        detail::DeviceImages images(configuration.device());
        std::vector<cf_sample> s = images.upload(all, [](const PixelInstance* p) -> const PixelInstance& { return *p; });
        const size_t F = ft.numFeatures(), T = ft.numThresholds();
        std::vector<WeightType> counters(F * T * numClasses * 2);
        detail::check(cf_histograms(images.get(), static_cast<int>(s.size()), s.data(), static_cast<int>(F),
                                    static_cast<int>(T), ft.features(), ft.thresholds(), static_cast<int>(numClasses),
                                    counters.data()));
        if (featureResponsesHost) {
            featureResponsesHost->assign(F * s.size(), 0.0);
            detail::check(cf_feature_responses(images.get(), static_cast<int>(s.size()), s.data(), static_cast<int>(F),
                                               ft.features(), featureResponsesHost->data()));
        }
        return counters;
    }

    // calculateScores (random_tree_image_gpu.cu:2137-2182): scores [T][F]
    std::vector<ScoreType> calculateScores(const std::vector<WeightType>& counters, const ImageFeaturesAndThresholds& ft,
                                           const std::vector<WeightType>& histogram) const {
        const size_t F = ft.numFeatures(), T = ft.numThresholds(), C = histogram.size();
        if (counters.size() != F * T * C * 2) throw std::runtime_error("calculateScores: counters size");
        std::vector<ScoreType> scores(T * F);
        detail::check(cf_scores(detail::context(configuration.device()), static_cast<int>(C), static_cast<int>(F),
                                static_cast<int>(T), counters.data(), histogram.data(), scores.data()));
        return scores;
    }

    // evaluateBestSplits (random_tree_image.cpp:239-502): one candidate table per level (seed drawn
    // from randomSource as there), every node's best split by the reference tie rule
    std::vector<SplitFunction<PixelInstance, ImageFeatureFunction>> evaluateBestSplits(
        RandomSource& randomSource,
        const std::vector<std::pair<std::shared_ptr<ImageTree>, std::vector<const PixelInstance*>>>& samplesPerNode) {
        std::vector<const PixelInstance*> all;
        std::vector<int64_t> offsets(1, 0);
        size_t C = 0;
        for (const auto& node : samplesPerNode) {
            all.insert(all.end(), node.second.begin(), node.second.end());
            offsets.push_back(static_cast<int64_t>(all.size()));
            C = std::max(C, node.first ? node.first->getNumClasses() : size_t(0));
        }
        if (C == 0) throw std::runtime_error("evaluateBestSplits: nodes need class histograms");
        const int seed = randomSource.uniformSampler(0xFFFFFF).getNext();
        detail::DeviceImages images(configuration.device());
        std::vector<cf_sample> s = images.upload(all, [](const PixelInstance* p) -> const PixelInstance& { return *p; });
        ImageFeaturesAndThresholds ft(configuration.getFeatureCount(), configuration.getThresholds());
        detail::check(cf_generate_features(images.get(), static_cast<int>(s.size()), s.data(),
                                           static_cast<uint32_t>(seed), static_cast<int>(ft.numFeatures()),
                                           static_cast<int>(ft.numThresholds()), configuration.getBoxRadius(),
                                           configuration.getRegionSize(), configuration.isUseDepthImages() ? 1 : 0,
                                           ft.features(), ft.thresholds()));
        std::vector<cf_split> best(samplesPerNode.size());
        detail::check(cf_evaluate_best_splits(images.get(), static_cast<int>(samplesPerNode.size()), offsets.data(),
                                              s.data(), static_cast<int>(C), static_cast<int>(ft.numFeatures()),
                                              static_cast<int>(ft.numThresholds()), ft.features(), ft.thresholds(),
                                              best.data()));
        std::vector<SplitFunction<PixelInstance, ImageFeatureFunction>> out;
        for (const cf_split& b : best)
            out.emplace_back(static_cast<size_t>(b.feature), ft.getFeatureFunction(static_cast<size_t>(b.feature)),
                             b.threshold, b.score);
        return out;
    }

    size_t getTreeId() const { return treeId; }

private:
    const size_t treeId;
    const TrainingConfiguration configuration;
};

// ---------------------------------------------------------------------------------------------
// RandomTreeImage (random_tree_image.h:1098-1189; random_tree_image.cpp:714-1059)
// ---------------------------------------------------------------------------------------------
class RandomTreeImage {
public:
    RandomTreeImage(int id, const TrainingConfiguration& configuration) : id(id), configuration(configuration) {}

    // a tree from the C-ABI (training or tree files); takes ownership of `handle`
    RandomTreeImage(cf_tree* handle, const TrainingConfiguration& configuration) : configuration(configuration) {
        adopt(handle);
    }

    // RandomTreeImage::train (random_tree_image.cpp:714-824): class prior, class- or pixel-uniform
    // sampling of subsampleCount pixels per image, block sort, breadth-first level training; the
    // sampling draws and the level seeds come from randomSource as there
    void train(const std::vector<LabeledRGBDImage>& trainLabelImages, RandomSource& randomSource,
               size_t subsampleCount, size_t numLabels) {
        trainFrom(trainLabelImages, randomSource.seedCounter(), static_cast<uint32_t>(subsampleCount), 1, 0, numLabels);
    }

    // RandomTreeImage::normalizeHistograms (random_tree_image.cpp:1061-1071) with the tree's prior
    void normalizeHistograms(const double histogramBias, const bool useLabelsPrior) {
        if (!tree) throw std::runtime_error("tree is not trained");
        tree->normalizeHistograms(classLabelPriorDistribution, histogramBias, useLabelsPrior);
    }

    const std::shared_ptr<ImageTree>& getTree() const { return tree; }
    const std::vector<WeightType>& getClassLabelPriorDistribution() const { return classLabelPriorDistribution; }
    size_t getId() const { return id; }
    const TrainingConfiguration& getConfiguration() const { return configuration; }
    bool shouldIgnoreLabel(const LabelType& label) const {
        for (const std::string& c : configuration.getIgnoredColors())
            if (LabelImage::encodeColor(RGBColor(c)) == label) return true;
        return false;
    }
    cf_tree* handle() const { return cfTree.get(); }

private:
    friend class RandomForestImage;

    // Sampling and training through the C-ABI. Pixels per image = samplesPerImage / numTrees; with
    // maxImages > 0 the tree first draws its image reservoir (random_forest_image.cpp:161-171). Both
    // draw from the seed counter, which is advanced as the reference advances its RandomSource.
    void trainFrom(const std::vector<LabeledRGBDImage>& trainLabelImages, int32_t& counter, uint32_t samplesPerImage,
                   int numTrees, int maxImages, size_t numLabels) {
        configuration.requireGpu();
        if (trainLabelImages.empty()) throw std::runtime_error("no training images");
        const int n = static_cast<int>(trainLabelImages.size());
        const int W = trainLabelImages[0].getWidth(), H = trainLabelImages[0].getHeight();
        const size_t plane = static_cast<size_t>(W) * H;
        std::vector<uint8_t> labels(plane * n);
        std::vector<uint16_t> depth(plane * n);
        std::vector<const RGBDImage*> images;
        LabelType maxLabel = 0;
        for (int i = 0; i < n; i++) {
            const LabeledRGBDImage& li = trainLabelImages[i];
            if (li.getWidth() != W || li.getHeight() != H)
                throw std::runtime_error("all images must have the same size (resize them to the largest frame)");
            const RGBDImage& im = li.getRGBDImage();
            if (!im.hasIntegratedDepth() || !im.hasIntegratedColor()) throw std::runtime_error("image is not integrated");
            images.push_back(&im);
            std::memcpy(&labels[plane * i], li.getLabelImage().data(), plane);
            // the pixels' own depths, recovered from the integral as PixelInstance does
            const int* sum = im.getDepthImage().data();
            const int* valid = sum + plane;
            for (int y = 0; y < H; y++)
                for (int x = 0; x < W; x++) {
                    auto at = [&](const int* a, int xx, int yy) -> uint32_t {
                        return (xx < 0 || yy < 0) ? 0u : static_cast<uint32_t>(a[static_cast<size_t>(yy) * W + xx]);
                    };
                    const uint32_t v = at(valid, x, y) - (at(valid, x - 1, y) + at(valid, x, y - 1) - at(valid, x - 1, y - 1));
                    const int mm = static_cast<int>(at(sum, x, y) - (at(sum, x - 1, y) + at(sum, x, y - 1) -
                                                                     at(sum, x - 1, y - 1)));
                    depth[plane * i + static_cast<size_t>(y) * W + x] =
                        (v == 1 && mm > 0) ? static_cast<uint16_t>(std::min(mm, 65535)) : 0;
                }
            for (size_t p = 0; p < plane; p++) maxLabel = std::max(maxLabel, labels[plane * i + p]);
        }
        const size_t C = numLabels ? numLabels : static_cast<size_t>(maxLabel) + 1;
        if (C > 256) throw std::runtime_error("at most 256 classes");
        detail::DeviceImages dev(configuration.device());
        dev.upload_images(images);
        const std::vector<uint8_t> ignored = detail::ignored_mask(configuration, C);
        cf_train_config cfg = configuration.toC();
        cfg.samples_per_image = samplesPerImage;
        cfg.max_images = maxImages;
        int32_t probe = counter;
        int64_t count = 0;
        std::vector<uint32_t> prior(C);
        detail::check(cf_sample_tree_pixels(n, W, H, labels.data(), depth.data(), static_cast<int>(C), ignored.data(),
                                            &cfg, numTrees, &probe, nullptr, 0, &count, nullptr));
        std::vector<cf_sample> samples(static_cast<size_t>(count));
        detail::check(cf_sample_tree_pixels(n, W, H, labels.data(), depth.data(), static_cast<int>(C), ignored.data(),
                                            &cfg, numTrees, &counter, samples.data(), count, &count, prior.data()));
        cf_tree* t = nullptr;
        detail::check(cf_train_tree(dev.get(), static_cast<int>(count), samples.data(), static_cast<int>(C), &cfg,
                                    static_cast<int>(id), &counter, CF_TRAIN_LEVEL_BATCHED, &t));
        detail::check(cf_tree_set_prior(t, prior.data(), static_cast<int>(C)));
        adopt(t);
    }

    void adopt(cf_tree* t) {
        cfTree.reset(t);
        int n = 0, C = 0, depth = 0, treeId = 0;
        detail::check(cf_tree_info(t, &n, &C, &depth, &treeId));
        id = static_cast<size_t>(treeId);
        tree = detail::build_tree(t);
        int count = 0;
        detail::check(cf_tree_prior(t, nullptr, 0, &count));
        std::vector<uint32_t> p(count);
        if (count) detail::check(cf_tree_prior(t, p.data(), count, &count));
        classLabelPriorDistribution.assign(p.begin(), p.end());
    }

    size_t id = 0;
    TrainingConfiguration configuration;
    std::shared_ptr<ImageTree> tree;
    std::vector<WeightType> classLabelPriorDistribution;
    detail::Handle<cf_tree> cfTree;
};

inline std::ostream& operator<<(std::ostream& os, const RandomTreeImage& tree) {
    os << "RandomTreeImage(id " << tree.getId();
    if (tree.getTree())
        os << ", " << tree.getTree()->countNodes() << " nodes, " << tree.getTree()->countLeafNodes() << " leaves, depth "
           << tree.getTree()->getTreeDepth();
    return os << ")";
}

// ---------------------------------------------------------------------------------------------
// Tree files (export.h, import.h): gzip-compressed JSON
// ---------------------------------------------------------------------------------------------
class RandomTreeExport {
public:
    RandomTreeExport(const TrainingConfiguration& configuration, const std::string& outputFolder,
                     const std::string& trainingFolder, bool verbose)
        : configuration(configuration), outputFolder(outputFolder), trainingFolder(trainingFolder), verbose(verbose) {}

    // <outputFolder>/tree<treeNr>.json.gz (export.cpp:292-313)
    void writeJSON(const RandomTreeImage& tree, size_t treeNr) const {
        if (!tree.handle()) throw std::runtime_error("tree is not trained");
        std::ostringstream path;
        path << outputFolder << "/tree" << treeNr << ".json.gz";
        const cf_train_config c = configuration.toC();
        const std::vector<WeightType>& prior = tree.getClassLabelPriorDistribution();
        detail::check(cf_tree_write_json(tree.handle(), &c, prior.empty() ? nullptr : prior.data(),
                                         path.str().c_str(), verbose ? 1 : 0));
    }
    template <class TreeEnsemble>
    void writeJSON(const TreeEnsemble& ensemble) const {
        for (size_t treeNr = 0; treeNr < ensemble.getTrees().size(); treeNr++)
            writeJSON(*(ensemble.getTree(treeNr)), treeNr);
    }

private:
    TrainingConfiguration configuration;
    std::string outputFolder, trainingFolder;
    bool verbose;
};

class RandomTreeImport {
public:
    // RandomTreeImport::readJSON (import.cpp:175-266): the configuration the tree was trained with
    static TrainingConfiguration readJSON(const std::string& filename, std::shared_ptr<RandomTreeImage>& tree) {
        cf_train_config c;
        std::vector<uint32_t> prior(256);
        cf_tree* t = nullptr;
        detail::check(cf_tree_read_json(filename.c_str(), &c, prior.data(), static_cast<int>(prior.size()), &t));
        const TrainingConfiguration configuration = TrainingConfiguration::fromC(c);
        tree = std::make_shared<RandomTreeImage>(t, configuration);
        return configuration;
    }
};

// ---------------------------------------------------------------------------------------------
// RandomForestImage (random_forest_image.h:44-168; random_forest_image.cpp)
// ---------------------------------------------------------------------------------------------
class RandomForestImage {
public:
    explicit RandomForestImage(const std::vector<std::string>& treeFiles,
                               const std::vector<int>& deviceIds = std::vector<int>(1, 0),
                               const AccelerationMode accelerationMode = GPU_ONLY, const double histogramBias = 0.0,
                               const bool useLabelsPrior = true) {
        if (treeFiles.empty()) throw std::runtime_error("cannot construct empty forest");
        std::vector<TrainingConfiguration> configurations;
        for (const std::string& f : treeFiles) {
            std::shared_ptr<RandomTreeImage> t;
            configurations.push_back(RandomTreeImport::readJSON(f, t));
            ensemble.push_back(t);
        }
        for (size_t i = 1; i < configurations.size(); i++)
            if (!configurations[0].equals(configurations[i], false))
                throw std::runtime_error("configurations of the trees differ");
        configuration = configurations[0];
        configuration.setDeviceIds(deviceIds);
        configuration.setAccelerationMode(accelerationMode);
        normalizeHistograms(histogramBias, useLabelsPrior);
    }

    explicit RandomForestImage(unsigned int treeCount, const TrainingConfiguration& configuration)
        : configuration(configuration), ensemble(treeCount) {
        if (treeCount == 0) throw std::runtime_error("a forest needs at least one tree");
    }

    explicit RandomForestImage(const std::vector<std::shared_ptr<RandomTreeImage>>& ensemble,
                               const TrainingConfiguration& configuration)
        : configuration(configuration), ensemble(ensemble) {
        if (ensemble.empty()) throw std::runtime_error("cannot construct empty forest");
    }

    // RandomForestImage::train (random_forest_image.cpp:132-182): SEED from the configured seed, tree
    // t trained from RandomSource(SEED + t) on the maxImages reservoir with samplesPerImage / treeCount
    // pixels per image. Trees train one after the other on the configuration's GPU.
    void train(const std::vector<LabeledRGBDImage>& trainLabelImages, size_t numLabels = 0,
               bool trainTreesSequentially = false) {
        (void)trainTreesSequentially;
        configuration.requireGpu();
        if (trainLabelImages.empty()) throw std::runtime_error("no training images");
        const size_t treeCount = ensemble.size();
        RandomSource randomSource(configuration.getRandomSeed());
        const int SEED = randomSource.uniformSampler(0xFFFF).getNext();
        for (size_t treeNr = 0; treeNr < treeCount; treeNr++) {
            auto tree = std::make_shared<RandomTreeImage>(static_cast<int>(treeNr), configuration);
            int32_t counter = SEED + static_cast<int>(treeNr);
            tree->trainFrom(trainLabelImages, counter, configuration.getSamplesPerImage(), static_cast<int>(treeCount),
                            configuration.getMaxImages(), numLabels);
            ensemble[treeNr] = tree;
        }
        forest.reset();
    }

    // RandomForestImage::predict (random_forest_image.cpp:258-352): per pixel the sum of the trees'
    // normalised leaf histograms, divided by its sum, and the label of the largest (lowest on ties);
    // probabilities (optional) receive [C][H][W]
    LabelImage predict(const RGBDImage& image, std::vector<float>* probabilities = nullptr, const bool onGPU = true,
                       bool useDepthImages = true) const {
        if (!onGPU) throw std::runtime_error("predict: this library predicts on the GPU only");
        (void)useDepthImages;
        if (!forest) throw std::runtime_error("histograms not normalized: call normalizeHistograms first");
        if (!image.hasIntegratedColor() || !image.hasIntegratedDepth()) throw std::runtime_error("image is not integrated");
        const size_t plane = static_cast<size_t>(image.getWidth()) * image.getHeight();
        LabelImage prediction(image.getWidth(), image.getHeight());
        detail::DeviceImages dev(configuration.device());
        dev.upload_images(std::vector<const RGBDImage*>(1, &image));
        if (probabilities) probabilities->assign(plane * getNumClasses(), 0.0f);
        detail::check(cf_predict_dataset_host(forest.get(), dev.get(), 0, 1,
                                              probabilities ? probabilities->data() : nullptr, prediction.data()));
        return prediction;
    }

    LabelType getNumClasses() const {
        LabelType numClasses = 0;
        for (const auto& tree : ensemble) {
            if (!tree || !tree->getTree()) throw std::runtime_error("tree is not trained");
            const LabelType c = static_cast<LabelType>(tree->getTree()->getNumClasses());
            if (numClasses == 0)
                numClasses = c;
            else if (c != numClasses)
                throw std::runtime_error("number of classes differ in trees");
        }
        return numClasses;
    }

    const std::shared_ptr<RandomTreeImage> getTree(size_t treeNr) const { return ensemble.at(treeNr); }
    const std::vector<std::shared_ptr<RandomTreeImage>>& getTrees() const { return ensemble; }
    const TrainingConfiguration& getConfiguration() const { return configuration; }

    bool shouldIgnoreLabel(const LabelType& label) const {
        for (const auto& tree : ensemble)
            if (tree && tree->shouldIgnoreLabel(label)) return true;
        return false;
    }

    std::map<LabelType, RGBColor> getLabelColorMap() const {
        std::map<LabelType, RGBColor> m;
        for (LabelType label = 0; label < getNumClasses(); label++) m[label] = LabelImage::decodeLabel(label);
        return m;
    }

    // RandomForestImage::normalizeHistograms (random_forest_image.cpp:366-376): every tree normalised
    // with its own prior, then packed for prediction (convertTree)
    void normalizeHistograms(const double histogramBias, const bool useLabelsPrior) {
        std::vector<cf_tree*> handles;
        for (const auto& tree : ensemble) {
            if (!tree || !tree->handle()) throw std::runtime_error("tree is not trained");
            tree->normalizeHistograms(histogramBias, useLabelsPrior);
            handles.push_back(tree->handle());
        }
        cf_forest* f = nullptr;
        detail::check(cf_forest_create(detail::context(configuration.device()), static_cast<int>(handles.size()),
                                       handles.data(), nullptr, histogramBias, useLabelsPrior ? 1 : 0, &f));
        forest.reset(f);
        detail::check(cf_forest_set_preprocessing(f, configuration.isUseDepthFilling() ? 1 : 0,
                                                  configuration.isUseCIELab() ? 1 : 0));
    }

    cf_forest* handle() const { return forest.get(); }

private:
    TrainingConfiguration configuration;
    std::vector<std::shared_ptr<RandomTreeImage>> ensemble;
    detail::Handle<cf_forest> forest;
};

// ---------------------------------------------------------------------------------------------
// Evaluation (predict.h, predict.cpp:45-207)
// ---------------------------------------------------------------------------------------------
class ConfusionMatrix {
public:
    ConfusionMatrix() : C(0), normalized(false) {}
    explicit ConfusionMatrix(size_t numClasses) : C(numClasses), data(numClasses * numClasses, 0.0), normalized(false) {}
    ConfusionMatrix(size_t numClasses, std::vector<LabelType> ignoredLabels)
        : C(numClasses), data(numClasses * numClasses, 0.0), normalized(false), ignoredLabels(ignoredLabels) {}

    void reset() {
        std::fill(data.begin(), data.end(), 0.0);
        normalized = false;
    }
    void resize(unsigned int numClasses) {
        C = numClasses;
        data.assign(static_cast<size_t>(C) * C, 0.0);
        normalized = false;
    }
    bool isNormalized() const { return normalized; }
    void operator+=(const ConfusionMatrix& o) {
        if (normalized) throw std::runtime_error("confusion matrix is already normalized");
        if (o.C != C) throw std::runtime_error("different number of classes in confusion matrix");
        for (size_t i = 0; i < data.size(); i++) data[i] += o.data[i];
    }
    double& operator()(int label, int prediction) { return data[static_cast<size_t>(label) * C + prediction]; }
    double operator()(int label, int prediction) const { return data[static_cast<size_t>(label) * C + prediction]; }
    void increment(int label, int prediction) {
        if (normalized) throw std::runtime_error("confusion matrix is already normalized");
        data[static_cast<size_t>(label) * C + prediction] += 1.0;
    }
    unsigned int getNumClasses() const { return static_cast<unsigned int>(C); }
    const std::vector<LabelType>& getIgnoredLabels() const { return ignoredLabels; }

    // ConfusionMatrix::normalize: rows divided by their sums (rows without pixels stay 0)
    void normalize() {
        if (normalized) throw std::runtime_error("confusion matrix is already normalized");
        std::vector<uint64_t> counts = toCounts();
        std::vector<double> norm(data.size());
        double avg = 0;
        detail::check(cf_confusion_average_class_accuracy(static_cast<int>(C), counts.data(), nullptr, 1, norm.data(),
                                                          &avg));
        data.swap(norm);
        normalized = true;
    }

    // averageClassAccuracy: the mean diagonal of the normalised matrix, ignored labels left out
    // unless includeVoid
    double averageClassAccuracy(bool includeVoid = true) const {
        std::vector<uint8_t> ignored(C, 0);
        for (LabelType l : ignoredLabels)
            if (l < C) ignored[l] = 1;
        if (normalized) {
            double total = 0;
            int n = 0;
            for (size_t l = 0; l < C; l++) {
                if (!includeVoid && ignored[l]) continue;
                total += data[l * C + l];
                n++;
            }
            return n ? total / n : 0.0;
        }
        std::vector<uint64_t> counts = toCounts();
        double avg = 0;
        detail::check(cf_confusion_average_class_accuracy(static_cast<int>(C), counts.data(), ignored.data(),
                                                          includeVoid ? 1 : 0, nullptr, &avg));
        return avg;
    }

private:
    std::vector<uint64_t> toCounts() const {
        std::vector<uint64_t> c(data.size());
        for (size_t i = 0; i < data.size(); i++) c[i] = static_cast<uint64_t>(data[i]);
        return c;
    }
    size_t C;
    std::vector<double> data;
    bool normalized;
    std::vector<LabelType> ignoredLabels;
};

// calculatePixelAccuracy (predict.cpp:148-207), counted on the GPU
inline double calculatePixelAccuracy(const LabelImage& prediction, const LabelImage& groundTruth,
                                     const bool includeVoid = true,
                                     const std::vector<LabelType>* ignoredLabels = nullptr,
                                     ConfusionMatrix* confusionMatrix = nullptr) {
    if (prediction.getWidth() != groundTruth.getWidth() || prediction.getHeight() != groundTruth.getHeight())
        throw std::runtime_error("prediction and ground truth have different sizes");
    const size_t plane = static_cast<size_t>(groundTruth.getWidth()) * groundTruth.getHeight();
    LabelType maxLabel = 0, maxPred = 0;
    for (size_t p = 0; p < plane; p++) {
        maxLabel = std::max(maxLabel, groundTruth.data()[p]);
        maxPred = std::max(maxPred, prediction.data()[p]);
    }
    size_t C = static_cast<size_t>(std::max(maxLabel, maxPred)) + 1;
    if (confusionMatrix) {
        if (confusionMatrix->getNumClasses() < static_cast<size_t>(maxLabel) + 1u) {
            confusionMatrix->resize(static_cast<unsigned int>(maxLabel) + 1u);
            confusionMatrix->reset();
        }
        C = std::max<size_t>(C, confusionMatrix->getNumClasses());
    }
    std::vector<uint8_t> ignored(C, 0);
    if (ignoredLabels)
        for (LabelType l : *ignoredLabels)
            if (l < C) ignored[l] = 1;
    std::vector<uint64_t> conf(confusionMatrix ? C * C : 0, 0);
    double accuracy = 0;
    if (plane == 0) return std::numeric_limits<double>::quiet_NaN();
    detail::check(cf_pixel_accuracy(detail::context(), 1, groundTruth.getWidth(), groundTruth.getHeight(),
                                    prediction.data(), groundTruth.data(), static_cast<int>(C), ignored.data(),
                                    includeVoid ? 1 : 0, confusionMatrix ? conf.data() : nullptr, &accuracy, 0));
    if (confusionMatrix) {
        if (confusionMatrix->isNormalized()) throw std::runtime_error("confusion matrix is already normalized");
        const size_t M = confusionMatrix->getNumClasses();
        for (size_t l = 0; l < C; l++)
            for (size_t p = 0; p < C; p++) {
                const uint64_t v = conf[l * C + p];
                if (!v) continue;
                if (l >= M || p >= M) throw std::runtime_error("prediction outside the confusion matrix's classes");
                (*confusionMatrix)(static_cast<int>(l), static_cast<int>(p)) += static_cast<double>(v);
            }
    }
    return accuracy;
}

}  // namespace curfil

#endif
