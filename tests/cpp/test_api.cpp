// Tests of the C++ interface (include/curfil_b200.hpp), written after the reference's own unit tests
// (src/tests/*.cpp, *.cu of deeplearningais/curfil): the same classes, calls and known answers.
//
//   test_api --group cpu       host-only behaviour (no GPU needed)
//   test_api --group nogpu     on a machine without a GPU: GPU work fails with std::runtime_error
//   test_api --group gpu       the known-answer and end-to-end tests on the GPU
//   test_api --sampler SEED LO HI COUNT    prints COUNT draws of Sampler(SEED, LO, HI)
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <iostream>
#include <string>
#include <unistd.h>
#include <vector>

#include "curfil_b200.hpp"

using namespace curfil;

namespace {

int g_checks = 0, g_failures = 0;

#define CHECK(cond)                                                                   \
    do {                                                                              \
        g_checks++;                                                                   \
        if (!(cond)) {                                                                \
            g_failures++;                                                             \
            std::fprintf(stderr, "%s:%d: CHECK(%s) failed\n", __FILE__, __LINE__, #cond); \
        }                                                                             \
    } while (0)

#define CHECK_EQ(a, b)                                                                          \
    do {                                                                                        \
        g_checks++;                                                                             \
        if (!((a) == (b))) {                                                                    \
            g_failures++;                                                                       \
            std::cerr << __FILE__ << ":" << __LINE__ << ": CHECK_EQ(" #a ", " #b ") failed: " << (a) \
                      << " vs " << (b) << std::endl;                                            \
        }                                                                                       \
    } while (0)

#define CHECK_CLOSE(a, b, tol)                                                                    \
    do {                                                                                          \
        g_checks++;                                                                               \
        const double va = (a), vb = (b);                                                          \
        if (!(std::fabs(va - vb) <= (tol))) {                                                     \
            g_failures++;                                                                         \
            std::cerr << __FILE__ << ":" << __LINE__ << ": CHECK_CLOSE(" #a ", " #b ") failed: " << va \
                      << " vs " << vb << std::endl;                                               \
        }                                                                                         \
    } while (0)

#define CHECK_THROWS(expr)                                                                      \
    do {                                                                                        \
        g_checks++;                                                                             \
        bool thrown = false;                                                                    \
        try {                                                                                   \
            expr;                                                                               \
        } catch (const std::runtime_error&) {                                                   \
            thrown = true;                                                                      \
        }                                                                                       \
        if (!thrown) {                                                                          \
            g_failures++;                                                                       \
            std::fprintf(stderr, "%s:%d: CHECK_THROWS(%s) did not throw\n", __FILE__, __LINE__, #expr); \
        }                                                                                       \
    } while (0)

struct Test {
    const char* group;
    const char* name;
    std::function<void()> fn;
};
std::vector<Test>& registry() {
    static std::vector<Test> t;
    return t;
}
struct Registrar {
    Registrar(const char* group, const char* name, std::function<void()> fn) { registry().push_back({group, name, fn}); }
};
#define TEST(group, name)                                   \
    static void name();                                     \
    static Registrar registrar_##name(#group, #name, name); \
    static void name()

TrainingConfiguration smallConfiguration(int seed = 4711, unsigned samplesPerImage = 500, unsigned features = 64,
                                         int maxDepth = 8) {
    return TrainingConfiguration(seed, samplesPerImage, features, 4, maxDepth, 20, 6, 10, 1, 0, 0, 50000, GPU_ONLY,
                                 false, false, std::vector<int>(1, 0), "classUniform", std::vector<std::string>(),
                                 true, false);
}

// ------------------------------------------------------------------------------------------ cpu
TEST(cpu, configuration) {
    // random_tree_test.cpp / train.cpp usage: the full constructor and its checks
    TrainingConfiguration a = smallConfiguration();
    CHECK_EQ(a.getRandomSeed(), 4711);
    CHECK_EQ(a.getFeatureCount(), 64u);
    CHECK_EQ(a.getSubsamplingType(), std::string("classUniform"));
    TrainingConfiguration b = a;
    CHECK(a == b);
    b.setRandomSeed(1);
    CHECK(a != b);                 // strict comparison includes the seed
    CHECK(a.equals(b, false));     // the non-strict one does not
    CHECK_THROWS(TrainingConfiguration(1, 1, 1, 1, 1, 1, 1, 1, 1, 5, 10, 1, GPU_ONLY));   // maxImages < cache
    CHECK_THROWS(TrainingConfiguration(1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 1, GPU_ONLY, true, false,
                                       std::vector<int>(1, 0), "classUniform", std::vector<std::string>(1, "")));
    CHECK_EQ(TrainingConfiguration::parseAccelerationModeString("gpu"), GPU_ONLY);
    CHECK_EQ(TrainingConfiguration::parseAccelerationModeString("cpu"), CPU_ONLY);
    CHECK_EQ(TrainingConfiguration::parseAccelerationModeString("compare"), GPU_AND_CPU_COMPARE);
    CHECK_THROWS(TrainingConfiguration::parseAccelerationModeString("tpu"));
    CHECK_EQ(a.getAccelerationModeString(), std::string("gpu"));
    const cf_train_config c = a.toC();
    CHECK_EQ(c.feature_count, 64u);
    CHECK_EQ(c.subsampling_type, 0);
    CHECK(TrainingConfiguration::fromC(c) == a);
    TrainingConfiguration p(1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 1, GPU_ONLY, true, false, std::vector<int>(1, 0),
                            "pixelUniform");
    CHECK_EQ(p.toC().subsampling_type, 1);
    TrainingConfiguration bad(1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 1, GPU_ONLY, true, false, std::vector<int>(1, 0), "x");
    CHECK_THROWS(bad.toC());
    // the CPU modes are refused, not silently run elsewhere
    TrainingConfiguration cpu = a;
    cpu.setAccelerationMode(CPU_ONLY);
    CHECK_THROWS(cpu.requireGpu());
    CHECK_THROWS(ImageFeatureEvaluation(0, cpu));
}

TEST(cpu, colors_and_labels) {
    // image_test.cpp: RGBColor parsing and the label colour registry
    RGBColor c("255,128,0");
    CHECK_EQ(int(c[0]), 255);
    CHECK_EQ(int(c[1]), 128);
    CHECK_EQ(int(c[2]), 0);
    CHECK_EQ(c.toString(), std::string("255,128,0"));
    CHECK_THROWS(RGBColor("256,0,0"));
    CHECK_THROWS(RGBColor("a,b,c"));
    CHECK_THROWS(RGBColor("1,2"));
    const LabelType l0 = LabelImage::encodeColor(RGBColor(1, 2, 3));
    const LabelType l1 = LabelImage::encodeColor(RGBColor(4, 5, 6));
    CHECK_EQ(int(l1), int(l0) + 1);
    CHECK_EQ(int(LabelImage::encodeColor(RGBColor(1, 2, 3))), int(l0));
    CHECK(LabelImage::decodeLabel(l1) == RGBColor(4, 5, 6));
    CHECK_THROWS(LabelImage::decodeLabel(250));

    LabelImage li(3, 2);
    li.setLabel(2, 1, 7);
    CHECK_EQ(int(li.getLabel(2, 1)), 7);
    CHECK_EQ(int(li.getLabel(0, 0)), 0);
    li.resizeImage(5, 4, 9);
    CHECK_EQ(int(li.getLabel(2, 1)), 7);
    CHECK_EQ(int(li.getLabel(4, 3)), 9);
    CHECK_EQ(int(li.getLabel(3, 0)), 9);
}

TEST(cpu, depth_and_xy) {
    CHECK_EQ(Depth(1.5).getIntValue(), 1500);
    CHECK(!Depth(0).isValid());
    CHECK(!Depth(std::numeric_limits<double>::quiet_NaN()).isValid());
    CHECK_THROWS(Depth(0).getFloatValue());
    // XY::normalize: int / float truncated toward zero (random_tree_image.h:82-87)
    const XY n = XY(10, -7).normalize(Depth(2000));
    CHECK_EQ(n.getX(), 5);
    CHECK_EQ(n.getY(), -3);
}

TEST(cpu, rgbd_image_storage) {
    RGBDImage im(3, 2);
    im.setColor(1, 1, 2, 0.5f);
    CHECK_EQ(im.getColor(1, 1, 2), 0.5f);
    im.setDepth(0, 1, Depth(1.25));
    CHECK_EQ(im.getDepth(0, 1).getIntValue(), 1250);
    CHECK_EQ(im.getDepthValid(0, 1), 1);
    im.setDepth(0, 1, Depth(0));              // invalid depth is stored as 0 (image.h:363-371)
    CHECK_EQ(im.getDepth(0, 1).getIntValue(), 0);
    CHECK_EQ(im.getDepthValid(0, 1), 0);
    im.setDepth(2, 0, Depth(2.0));
    im.resizeImage(5, 4);                      // RGBDImage::resizeImage: NaN colour, zero depth outside
    CHECK_EQ(im.getColor(1, 1, 2), 0.5f);
    CHECK(std::isnan(im.getColor(4, 3, 0)));
    CHECK_EQ(im.getDepth(2, 0).getIntValue(), 2000);
    CHECK_EQ(im.getDepth(4, 3).getIntValue(), 0);
    CHECK_EQ(im.getDepthValid(4, 3), 0);
    CHECK_THROWS(PixelInstance(&im, 0, 1, 1));  // not integrated
    auto a = std::make_shared<RGBDImage>(3, 2);
    auto b = std::make_shared<LabelImage>(4, 2);
    CHECK_THROWS(LabeledRGBDImage(a, b));
}

TEST(cpu, feature_function) {
    // random_tree_image.h:404-460: constructor check, sort key, table round trip
    CHECK_THROWS(ImageFeatureFunction(DEPTH, Offset(1, 1), Region(2, 2), 0, Offset(1, 1), Region(1, 1), 0));
    ImageFeatureFunction f(COLOR, Offset(-3, 4), Region(2, 1), 1, Offset(5, -6), Region(3, 3), 2);
    int8_t col[11];
    f.toColumn(col);
    CHECK(ImageFeatureFunction::fromColumn(col) == f);
    const int key = (1 << 30) | (1 << 26) | (2 << 22) | ((4 + 127) << 14) | ((-3 + 127) << 6);
    CHECK_EQ(f.getSortKey(), key);
    ImageFeaturesAndThresholds ft(4, 3);
    ft.setFeatureFunction(2, f);
    ft.setThreshold(1, 2, 7.5f);
    CHECK(ft.getFeatureFunction(2) == f);
    CHECK_EQ(ft.getThreshold(1, 2), 7.5);
    CHECK_EQ(int(ft.types()[2]), int(COLOR));
    CHECK_EQ(int(ft.offset2Y()[2]), -6);
    CHECK_EQ(int(ft.channel2()[2]), 2);
}

TEST(cpu, confusion_matrix_host) {
    ConfusionMatrix m(3);
    m.increment(0, 0);
    m.increment(0, 1);
    m.increment(2, 2);
    CHECK_EQ(m(0, 1), 1.0);
    ConfusionMatrix other(3);
    other.increment(1, 1);
    m += other;
    CHECK_EQ(m(1, 1), 1.0);
    ConfusionMatrix wrong(2);
    CHECK_THROWS(m += wrong);
}

// ------------------------------------------------------------------------------------------ nogpu
TEST(nogpu, gpu_work_fails_loudly) {
    RGBDImage im(4, 4);
    CHECK_THROWS(im.calculateIntegral());
}

// ------------------------------------------------------------------------------------------ gpu
TEST(gpu, integral_kats) {
    // image_test.cpp:87-133: colour 3x3
    const float px[3][3] = {{5, 2, 3}, {1, 5, 4}, {2, 2, 1}};
    const float in[3][3] = {{5, 7, 10}, {6, 13, 20}, {8, 17, 25}};
    RGBDImage a(3, 3);
    for (int y = 0; y < 3; y++)
        for (int x = 0; x < 3; x++)
            for (int c = 0; c < 3; c++) a.setColor(x, y, c, px[y][x]);
    a.calculateIntegral();
    CHECK_THROWS(a.calculateIntegral());       // "image already integrated"
    for (int y = 0; y < 3; y++)
        for (int x = 0; x < 3; x++)
            for (int c = 0; c < 3; c++) CHECK_EQ(a.getColor(x, y, c), in[y][x]);
    // image_test.cpp:135-162: 640x480 of 255, a 20x16 box
    RGBDImage big(640, 480);
    for (int y = 0; y < 480; y++)
        for (int x = 0; x < 640; x++)
            for (int c = 0; c < 3; c++) big.setColor(x, y, c, 255.0f);
    big.calculateIntegral();
    const int x = 640 - 11, y = 480 - 9;
    for (int c = 0; c < 3; c++) {
        const double s = double(big.getColor(x + 10, y + 8, c)) - big.getColor(x + 10, y - 8, c) -
                         big.getColor(x - 10, y + 8, c) + big.getColor(x - 10, y - 8, c);
        CHECK_EQ(s, 20.0 * 16.0 * 255.0);
    }
    // image_test.cpp:164-279: depth 3x2, the second write to (0,1) wins
    RGBDImage d(3, 2);
    d.setDepth(0, 0, Depth(5.0));
    d.setDepth(0, 1, Depth(15.0));
    d.setDepth(0, 1, Depth(10.0));
    d.setDepth(1, 0, Depth(35.0));
    d.setDepth(2, 1, Depth(10.0));
    d.calculateIntegral();
    const int sums[2][3] = {{5000, 40000, 40000}, {15000, 50000, 60000}};
    const int valid[2][3] = {{1, 2, 2}, {2, 3, 4}};
    for (int yy = 0; yy < 2; yy++)
        for (int xx = 0; xx < 3; xx++) {
            CHECK_EQ(d.getDepth(xx, yy).getIntValue(), sums[yy][xx]);
            CHECK_EQ(d.getDepthValid(xx, yy), valid[yy][xx]);
        }
    // PixelInstance recovers the pixel's own depth (random_tree_image.h:140-165)
    CHECK_EQ(PixelInstance(&d, 0, 0, 1).getDepth().getIntValue(), 10000);
    CHECK_EQ(PixelInstance(&d, 0, 1, 0).getDepth().getIntValue(), 35000);
    CHECK(!PixelInstance(&d, 0, 1, 1).getDepth().isValid());
}

TEST(gpu, fill_depth_kat) {
    // image_test.cpp:425-456
    RGBDImage im(200, 100);
    im.setDepth(20, 30, Depth(1.5));
    im.setDepth(30, 20, Depth(2.5));
    im.fillDepth();
    bool ok = true;
    for (int y = 0; y < 100; y++)
        for (int x = 0; x < 200; x++) {
            const int want = y < 30 ? 2500 : 1500;
            ok = ok && im.getDepth(x, y).getIntValue() == want && im.getDepthValid(x, y) == 1;
        }
    CHECK(ok);
}

TEST(gpu, depth_feature_kat) {
    // random_tree_image_gpu_test.cu:318-488
    const int W = 16, H = 20;
    RGBDImage im(W, H);
    im.setDepth(7, 3, Depth(1.5));
    im.setDepth(7, 4, Depth(1.7));
    im.setDepth(8, 4, Depth(4.5));
    im.setDepth(3, 2, Depth(3.9));
    im.calculateIntegral();
    ImageFeatureFunction f(DEPTH, Offset(1, 1), Region(2, 2), 0, Offset(-3, -1), Region(1, 1), 0);
    PixelInstance s0(&im, 0, Depth(1.0), 6, 3), s1(&im, 1, Depth(1.0), 6, 3);
    CHECK_CLOSE(f.calculateFeatureResponse(s0), (1.5 + 1.7 + 4.5) / 3 - 3.9, 1e-8);
    TrainingConfiguration cfg = smallConfiguration();
    ImageFeatureEvaluation eval(0, cfg);
    ImageFeaturesAndThresholds ft(1, 100);
    ft.setFeatureFunction(0, f);
    for (int t = 0; t < 100; t++) ft.setThreshold(t, 0, (t - 50) / 10.0f);
    std::vector<std::vector<const PixelInstance*>> batches(1, std::vector<const PixelInstance*>{&s0, &s1});
    std::vector<WeightType> counters = eval.calculateFeatureResponsesAndHistograms(2, batches, ft);
    bool ok = true;
    for (int label = 0; label < 2; label++)
        for (int t = 0; t < 100; t++) {
            const WeightType left = counters[(t * 2 + label) * 2 + 0], right = counters[(t * 2 + label) * 2 + 1];
            ok = ok && left == WeightType(t >= 37) && left + right == 1;
        }
    CHECK(ok);
}

TEST(gpu, color_feature_complex_kat) {
    // random_tree_image_gpu_test.cu:653-866: two images, v = 100 c + y W + x and its half
    const int W = 12, H = 15;
    RGBDImage a(W, H), b(W, H);
    for (int c = 0; c < 3; c++)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) {
                const float v = 100.0f * c + y * W + x;
                a.setColor(x, y, c, v);
                b.setColor(x, y, c, v / 2.0f);
            }
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            a.setDepth(x, y, Depth(1.0));
            b.setDepth(x, y, Depth(1.0));
        }
    a.calculateIntegral();
    b.calculateIntegral();
    CHECK_EQ(a.getColor(W - 1, H - 1, 0), 16110.0f);
    CHECK_EQ(a.getColor(W - 1, H - 1, 1), 34110.0f);
    CHECK_EQ(a.getColor(W - 1, H - 1, 2), 52110.0f);
    const ImageFeatureFunction f[3] = {
        ImageFeatureFunction(COLOR, Offset(2, -1), Region(2, 1), 0, Offset(-3, 4), Region(1, 2), 2),
        ImageFeatureFunction(COLOR, Offset(2, -1), Region(2, 2), 1, Offset(-3, 4), Region(1, 1), 2),
        ImageFeatureFunction(COLOR, Offset(-2, 1), Region(3, 1), 1, Offset(3, -4), Region(3, 3), 0)};
    const PixelInstance s[4] = {PixelInstance(&a, 0, Depth(1.0), 6, 4), PixelInstance(&b, 0, Depth(2.0), 6, 4),
                                PixelInstance(&a, 1, Depth(1.5), 5, 5), PixelInstance(&b, 1, Depth(3.1), 3, 4)};
    const double want[3][4] = {{-2040, -444, -884, -424}, {1186, -244, -484, -224}, {NAN, 244, 572, 224}};
    std::vector<PixelInstance> all(s, s + 4);
    for (int i = 0; i < 3; i++) {
        std::vector<FeatureResponseType> r = f[i].calculateFeatureResponses(all);
        for (int j = 0; j < 4; j++) {
            if (std::isnan(want[i][j]))
                CHECK(std::isnan(r[j]));
            else
                CHECK_EQ(r[j], want[i][j]);
        }
    }
    ImageFeaturesAndThresholds ft(3, 2);
    const float thr[2][3] = {{0.0f, -300.0f, 0.0f}, {-500.0f, 0.0f, 500.0f}};
    for (int i = 0; i < 3; i++) {
        ft.setFeatureFunction(i, f[i]);
        for (int t = 0; t < 2; t++) ft.setThreshold(t, i, thr[t][i]);
    }
    ImageFeatureEvaluation eval(0, smallConfiguration());
    std::vector<std::vector<const PixelInstance*>> batches(1, std::vector<const PixelInstance*>{&s[0], &s[1], &s[2], &s[3]});
    std::vector<WeightType> counters = eval.calculateFeatureResponsesAndHistograms(2, batches, ft);
    // counters(feat, thresh, label, side)
    const int expect[3][2][2][2] = {{{{2, 0}, {2, 0}}, {{1, 1}, {1, 1}}},
                                    {{{0, 2}, {1, 1}}, {{1, 1}, {2, 0}}},
                                    {{{0, 2}, {0, 2}}, {{1, 1}, {1, 1}}}};
    for (int i = 0; i < 3; i++)
        for (int t = 0; t < 2; t++)
            for (int l = 0; l < 2; l++)
                for (int side = 0; side < 2; side++)
                    CHECK_EQ(int(counters[((i * 2 + t) * 2 + l) * 2 + side]), expect[i][t][l][side]);
}

TEST(gpu, score_kats) {
    // random_tree_image_gpu_test.cu:106-240 through calculateScores
    struct Kat {
        std::vector<WeightType> left, right, all;
        double expected, rel;
    };
    const std::vector<Kat> kats = {
        {{5, 8}, {3, 1}, {8, 9}, 0.080185, 1e-6},
        {{2, 8}, {6, 1}, {8, 9}, 0.33339, 1e-5},
        {{56, 241, 290, 3, 18}, {30, 0, 1, 0, 249}, {86, 241, 291, 3, 267}, 0.491311, 1e-5},
        {{50, 100, 0, 0, 0}, {0, 0, 50, 0, 100}, {50, 100, 50, 0, 100}, 0.68533, 1e-5}};
    ImageFeatureEvaluation eval(0, smallConfiguration());
    for (const Kat& k : kats) {
        const size_t C = k.all.size();
        ImageFeaturesAndThresholds ft(1, 1);
        std::vector<WeightType> counters(C * 2);
        for (size_t c = 0; c < C; c++) {
            counters[c * 2 + 0] = k.left[c];
            counters[c * 2 + 1] = k.right[c];
        }
        const std::vector<ScoreType> s = eval.calculateScores(counters, ft, k.all);
        CHECK_CLOSE(s[0], k.expected, k.expected * k.rel);
    }
    // :114-158: the reference checks its GPU scores within 1e-6 percent of these
    for (WeightType num = 1; num < 10; num++) {
        ImageFeaturesAndThresholds ft(1, 1);
        CHECK_EQ(eval.calculateScores({num, num, num, num}, ft, {2 * num, 2 * num})[0], 0.0);
        CHECK_CLOSE(eval.calculateScores({0, 2 * num, 2 * num, 0}, ft, {2 * num, 2 * num})[0], 1.0, 1e-12);
    }
}

TEST(gpu, normalize_histogram_kats) {
    // random_tree_test.cpp:46-154 through RandomTree::normalizeHistograms
    struct Kat {
        std::vector<WeightType> hist, prior;
        double bias;
        std::vector<double> expected;
    };
    const std::vector<Kat> kats = {
        {{850, 50, 100}, {100, 100, 100}, 0.0, {0.850 / 3.0, 0.050 / 3.0, 0.100 / 3.0}},
        {{50, 50, 50}, {80, 10, 10}, 0.0, {(1 / 3.0) * 0.8, (1 / 3.0) * 0.1, (1 / 3.0) * 0.1}},
        {{50, 50, 50}, {80, 10, 10}, 0.5, {0.0, 0.0, 0.0}},
        {{60, 20, 20}, {50, 25, 25}, 0.5, {0.5, 0.0, 0.0}},
        {{20, 40, 40}, {20, 10, 10}, 0.2, {0.0, 0.5 * 0.25, 0.5 * 0.25}}};
    for (const Kat& k : kats) {
        ImageTree leaf(0, 1, k.hist);
        leaf.normalizeHistograms(k.prior, k.bias, true);
        for (size_t c = 0; c < 3; c++) CHECK_CLOSE(leaf.getNormalizedHistogram()[c], k.expected[c], 1e-12);
    }
}

// frames of the library's seeded synthetic scene generator as LabeledRGBDImages
struct Frames {
    int n, W, H;
    std::vector<uint8_t> rgb, labels;
    std::vector<uint16_t> depth;
    std::vector<LabeledRGBDImage> images;
};

Frames makeFrames(uint64_t seed, int n, int W, int H, int cells, int classes) {
    Frames f{n, W, H, {}, {}, {}, {}};
    const size_t plane = static_cast<size_t>(W) * H;
    f.rgb.resize(plane * 3 * n);
    f.depth.resize(plane * n);
    f.labels.resize(plane * n);
    detail::check(cf_synthetic_frames(seed, n, W, H, cells, classes, -1, f.rgb.data(), f.depth.data(), f.labels.data()));
    for (int i = 0; i < n; i++) {
        auto im = std::make_shared<RGBDImage>(
            RGBDImage::fromRaw(W, H, &f.rgb[plane * 3 * i], &f.depth[plane * i]));
        im->calculateIntegral();
        auto li = std::make_shared<LabelImage>(W, H);
        std::memcpy(li->data(), &f.labels[plane * i], plane);
        f.images.emplace_back(im, li);
    }
    return f;
}

struct TreeArrays {
    std::vector<int32_t> level, left, featureId;
    std::vector<int8_t> feature;
    std::vector<float> threshold;
    std::vector<double> score;
    std::vector<uint32_t> hist;
};

TreeArrays exportTree(cf_tree* t) {
    int n = 0, C = 0, depth = 0, id = 0;
    detail::check(cf_tree_info(t, &n, &C, &depth, &id));
    TreeArrays a;
    a.level.resize(n);
    a.left.resize(n);
    a.featureId.resize(n);
    a.feature.resize(static_cast<size_t>(n) * 11);
    a.threshold.resize(n);
    a.score.resize(n);
    a.hist.resize(static_cast<size_t>(n) * C);
    detail::check(cf_tree_export(t, a.level.data(), a.left.data(), a.feature.data(), a.threshold.data(), a.score.data(),
                                 a.featureId.data(), a.hist.data(), nullptr));
    return a;
}

bool sameSplits(const TreeArrays& a, const TreeArrays& b) {
    if (a.left != b.left || a.hist != b.hist || a.level != b.level) return false;
    for (size_t i = 0; i < a.left.size(); i++) {
        if (a.left[i] < 0) continue;
        if (a.threshold[i] != b.threshold[i] || a.featureId[i] != b.featureId[i]) return false;
        if (std::memcmp(&a.feature[i * 11], &b.feature[i * 11], 11) != 0) return false;
    }
    return true;
}

TEST(gpu, forest_train_predict_export_import) {
    // random_forest_image_test / import_export_test: train, predict, write and read back
    const int C = 6, T = 3;
    Frames f = makeFrames(11, 4, 80, 60, 10, C);
    TrainingConfiguration cfg = smallConfiguration(4711, 600, 96, 10);
    RandomForestImage forest(T, cfg);
    forest.train(f.images, C);
    CHECK_EQ(int(forest.getNumClasses()), C);

    // the same forest through the C-ABI's RandomForestImage::train on the raw frames
    cf_context* ctx = detail::context();
    std::vector<cf_tree*> ref(T, nullptr);
    const cf_train_config c = cfg.toC();
    detail::check(cf_forest_train(ctx, f.n, f.W, f.H, f.rgb.data(), f.depth.data(), f.labels.data(), C, nullptr, &c, T,
                                  CF_TRAIN_LEVEL_BATCHED, ref.data()));
    for (int t = 0; t < T; t++) {
        CHECK(sameSplits(exportTree(forest.getTree(t)->handle()), exportTree(ref[t])));
        CHECK(forest.getTree(t)->getClassLabelPriorDistribution().size() == size_t(C));
        CHECK(forest.getTree(t)->getTree()->countNodes() > 1);
    }

    CHECK_THROWS(forest.predict(f.images[0].getRGBDImage()));   // histograms not normalised yet
    forest.normalizeHistograms(0.0, true);
    cf_forest* refForest = nullptr;
    detail::check(cf_forest_create(ctx, T, ref.data(), nullptr, 0.0, 1, &refForest));
    const size_t plane = static_cast<size_t>(f.W) * f.H;
    double accuracy = 0;
    ConfusionMatrix confusion(C);
    for (int i = 0; i < f.n; i++) {
        std::vector<float> probs;
        LabelImage pred = forest.predict(f.images[i].getRGBDImage(), &probs);
        std::vector<float> refProbs(plane * C);
        std::vector<uint8_t> refLabels(plane);
        detail::check(cf_predict_host(refForest, 1, f.W, f.H, &f.rgb[plane * 3 * i], &f.depth[plane * i],
                                      refProbs.data(), refLabels.data()));
        CHECK(std::memcmp(pred.data(), refLabels.data(), plane) == 0);
        CHECK(probs == refProbs);
        // the leaf path of one pixel: RandomTree::classifySoft agrees with the packed forest's leaf
        const PixelInstance px(&f.images[i].getRGBDImage(), 0, static_cast<uint16_t>(f.W / 2),
                               static_cast<uint16_t>(f.H / 2));
        const std::vector<double>& leaf = forest.getTree(0)->getTree()->classifySoft(px);
        CHECK_EQ(leaf.size(), size_t(C));
        accuracy += calculatePixelAccuracy(pred, f.images[i].getLabelImage(), true, nullptr, &confusion);
    }
    accuracy /= f.n;
    CHECK(accuracy > 0.5);
    double total = 0;
    for (int l = 0; l < C; l++)
        for (int p = 0; p < C; p++) total += confusion(l, p);
    CHECK_EQ(total, double(plane * f.n));
    const double avg = confusion.averageClassAccuracy(true);
    CHECK(avg > 0.3 && avg <= 1.0);

    // export and import (import_export_test.cpp:103-167): the read forest predicts the same
    char dir[] = "/tmp/curfil_cpp_XXXXXX";
    CHECK(mkdtemp(dir) != nullptr);
    RandomTreeExport exporter(cfg, dir, "synthetic", false);
    exporter.writeJSON(forest);
    std::vector<std::string> files;
    for (int t = 0; t < T; t++) files.push_back(std::string(dir) + "/tree" + std::to_string(t) + ".json.gz");
    RandomForestImage read(files);
    CHECK(read.getConfiguration().equals(cfg, false));
    for (int t = 0; t < T; t++) CHECK(sameSplits(exportTree(read.getTree(t)->handle()), exportTree(ref[t])));
    LabelImage p0 = forest.predict(f.images[0].getRGBDImage());
    LabelImage p1 = read.predict(f.images[0].getRGBDImage());
    CHECK(std::memcmp(p0.data(), p1.data(), plane) == 0);
    for (int t = 0; t < T; t++) std::remove(files[t].c_str());
    rmdir(dir);

    cf_forest_destroy(refForest);
    for (cf_tree* t : ref) cf_tree_destroy(t);
}

TEST(gpu, evaluate_best_splits_matches_histograms_and_scores) {
    // random_tree_image_gpu_test.cu compare style: evaluateBestSplits equals the argmax over
    // calculateFeatureResponsesAndHistograms + calculateScores with the reference tie rule
    const int C = 5;
    Frames f = makeFrames(5, 2, 64, 48, 8, C);
    TrainingConfiguration cfg = smallConfiguration(1, 500, 48, 6);
    ImageFeatureEvaluation eval(0, cfg);
    std::mt19937 rng(3);
    std::vector<PixelInstance> pixels;
    for (int i = 0; i < 700; i++) {
        const int img = static_cast<int>(rng() % 2);
        const uint16_t x = static_cast<uint16_t>(rng() % f.W), y = static_cast<uint16_t>(rng() % f.H);
        const LabelType label = f.images[img].getLabelImage().getLabel(x, y);
        pixels.emplace_back(&f.images[img].getRGBDImage(), label, x, y);
    }
    std::vector<std::pair<std::shared_ptr<ImageTree>, std::vector<const PixelInstance*>>> nodes(2);
    for (int n = 0; n < 2; n++) {
        std::vector<WeightType> hist(C, 0);
        const size_t lo = n == 0 ? 0 : 450, hi = n == 0 ? 450 : pixels.size();
        for (size_t i = lo; i < hi; i++) {
            nodes[n].second.push_back(&pixels[i]);
            hist[pixels[i].getLabel()]++;
        }
        nodes[n].first = std::make_shared<ImageTree>(n, 1, hist);
    }
    RandomSource rs1(77), rs2(77);
    const std::vector<SplitFunction<PixelInstance, ImageFeatureFunction>> best = eval.evaluateBestSplits(rs1, nodes);
    const int seed = rs2.uniformSampler(0xFFFFFF).getNext();
    std::vector<const PixelInstance*> all;
    for (auto& n : nodes) all.insert(all.end(), n.second.begin(), n.second.end());
    ImageFeaturesAndThresholds ft = eval.generateRandomFeatures(all, seed, true);
    for (int n = 0; n < 2; n++) {
        std::vector<std::vector<const PixelInstance*>> batches(1, nodes[n].second);
        std::vector<WeightType> counters = eval.calculateFeatureResponsesAndHistograms(C, batches, ft);
        std::vector<ScoreType> scores = eval.calculateScores(counters, ft, nodes[n].first->getHistogram());
        // thresholds outer, features inner; replace only when better by >= 1e-13 (random_tree.cpp:36-52)
        double bestScore = -std::numeric_limits<double>::infinity();
        size_t bf = 0, bt = 0;
        for (size_t t = 0; t < ft.numThresholds(); t++)
            for (size_t fi = 0; fi < ft.numFeatures(); fi++) {
                const double s = scores[t * ft.numFeatures() + fi];
                if (s > bestScore && std::fabs(s - bestScore) >= 1e-13) {
                    bestScore = s;
                    bf = fi;
                    bt = t;
                }
            }
        CHECK(bestScore > 0.0);
        CHECK_CLOSE(best[n].getScore(), bestScore, 1e-12 * std::max(1.0, bestScore));
        CHECK(best[n].getFeature() == ft.getFeatureFunction(best[n].getFeatureId()));
        // the chosen (feature, threshold) is the sequential choice, or ties with it within 1e-6
        const size_t f = best[n].getFeatureId();
        bool found = false;
        for (size_t t = 0; t < ft.numThresholds(); t++) {
            if (static_cast<float>(ft.getThreshold(t, f)) != best[n].getThreshold()) continue;
            const double s = scores[t * ft.numFeatures() + f];
            found = found || (f == bf && t == bt) || std::fabs(s - bestScore) <= 1e-6 * std::max(1.0, bestScore);
        }
        CHECK(found);
    }
}

int runGroup(const std::string& group) {
    int ran = 0;
    for (const Test& t : registry()) {
        if (group != t.group) continue;
        const int before = g_failures;
        try {
            t.fn();
        } catch (const std::exception& e) {
            g_failures++;
            std::fprintf(stderr, "%s: uncaught exception: %s\n", t.name, e.what());
        }
        std::printf("%s %s\n", g_failures == before ? "PASS" : "FAIL", t.name);
        ran++;
    }
    std::printf("%d tests, %d checks, %d failures\n", ran, g_checks, g_failures);
    return (ran > 0 && g_failures == 0) ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc == 3 && std::string(argv[1]) == "--group") return runGroup(argv[2]);
    if (argc == 6 && std::string(argv[1]) == "--sampler") {
        Sampler s(std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4]));
        const int count = std::atoi(argv[5]);
        for (int i = 0; i < count; i++) std::printf("%d\n", s.getNext());
        return 0;
    }
    std::fprintf(stderr, "usage: %s --group cpu|nogpu|gpu | --sampler SEED LO HI COUNT\n", argv[0]);
    return 2;
}
