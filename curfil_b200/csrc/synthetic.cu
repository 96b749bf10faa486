// Seeded synthetic RGB-D scenes standing in for recorded frames (no dataset is available offline).
//
// Every frame is a Voronoi partition into `num_cells` cells. Each cell takes a class; each class
// has a fixed base colour and depth range shared by all frames, so the task is learnable. Colour:
// uint8 RGB, the cell colour plus Gaussian noise (sigma 8). Depth: uint16 mm, a plane per cell
// clamped to [500, 5000], with 10% of the pixels set to 0 (missing). Labels: the cell class with
// 5% of the pixels flipped uniformly to another class. Frames are independent (seed, frame index)
// streams, so the output does not depend on the number of host threads.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "internal.h"

namespace {

struct SplitMix {
    uint64_t s;
    explicit SplitMix(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    int below(int n) { return static_cast<int>(uniform() * n); }
    double normal() {
        // Box-Muller
        double u1 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        const double u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

void make_frame(uint64_t seed, int img, int W, int H, int K, int C, int void_class, const std::vector<double>& cls_rgb,
                const std::vector<double>& cls_depth, uint8_t* rgb, uint16_t* depth, uint8_t* labels) {
    SplitMix rng(seed * 0x100000001B3ull + static_cast<uint64_t>(img) * 0x9E3779B97F4A7C15ull + 17);
    std::vector<double> sx(K), sy(K);
    std::vector<int> cls(K);
    std::vector<double> col(3 * K), a(K), bx(K), by(K);
    for (int k = 0; k < K; k++) {
        sx[k] = rng.uniform() * W;
        sy[k] = rng.uniform() * H;
        cls[k] = rng.below(C);
        for (int c = 0; c < 3; c++) col[3 * k + c] = cls_rgb[3 * cls[k] + c] + (rng.uniform() - 0.5) * 30.0;
        a[k] = cls_depth[cls[k]] + (rng.uniform() - 0.5) * 600.0;
        bx[k] = (rng.uniform() - 0.5) * 4.0;
        by[k] = (rng.uniform() - 0.5) * 4.0;
    }
    (void)void_class;
    for (int y = 0; y < H; y++) {
        for (int x = 0; x < W; x++) {
            int best = 0;
            double bd = 1e300;
            for (int k = 0; k < K; k++) {
                const double dx = x - sx[k], dy = y - sy[k];
                const double d = dx * dx + dy * dy;
                if (d < bd) {
                    bd = d;
                    best = k;
                }
            }
            const size_t p = static_cast<size_t>(y) * W + x;
            for (int c = 0; c < 3; c++) {
                const double v = col[3 * best + c] + 8.0 * rng.normal();
                rgb[p * 3 + c] = static_cast<uint8_t>(std::min(255.0, std::max(0.0, std::round(v))));
            }
            double d = a[best] + bx[best] * (x - sx[best]) + by[best] * (y - sy[best]);
            d = std::min(5000.0, std::max(500.0, d));
            depth[p] = rng.uniform() < 0.1 ? 0 : static_cast<uint16_t>(std::lround(d));
            int label = cls[best];
            if (C > 1 && rng.uniform() < 0.05) {
                int other = rng.below(C - 1);
                if (other >= label) other++;
                label = other;
            }
            labels[p] = static_cast<uint8_t>(label);
        }
    }
}

}  // namespace

extern "C" cf_status cf_synthetic_frames(uint64_t seed, int num_images, int width, int height, int num_cells,
                                         int num_classes, int void_class, uint8_t* rgb, uint16_t* depth_mm,
                                         uint8_t* labels) {
    return cf_synthetic_frames_from(seed, 0, num_images, width, height, num_cells, num_classes, void_class, rgb,
                                    depth_mm, labels);
}

extern "C" cf_status cf_synthetic_frames_from(uint64_t seed, int first_index, int num_images, int width, int height,
                                              int num_cells, int num_classes, int void_class, uint8_t* rgb,
                                              uint16_t* depth_mm, uint8_t* labels) {
    return cf::guard([&] {
        CF_REQUIRE(rgb && depth_mm && labels, "cf_synthetic_frames: NULL argument");
        CF_REQUIRE(first_index >= 0, "cf_synthetic_frames: negative first frame index");
        CF_REQUIRE(num_images >= 1 && width >= 1 && height >= 1 && num_cells >= 1, "cf_synthetic_frames: empty");
        CF_REQUIRE(num_classes >= 1 && num_classes <= 256, "cf_synthetic_frames: classes must be in [1, 256]");
        // class appearance shared by all frames
        SplitMix crng(seed ^ 0xC1A55E5ull);
        std::vector<double> cls_rgb(3 * num_classes), cls_depth(num_classes);
        for (int c = 0; c < num_classes; c++) {
            for (int k = 0; k < 3; k++) cls_rgb[3 * c + k] = 30.0 + 195.0 * crng.uniform();
            cls_depth[c] = 900.0 + 3600.0 * crng.uniform();
        }
        const size_t plane = static_cast<size_t>(width) * height;
        unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        nt = std::min<unsigned>(nt, static_cast<unsigned>(num_images));
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nt; t++) {
            pool.emplace_back([&, t] {
                for (int i = static_cast<int>(t); i < num_images; i += static_cast<int>(nt))
                    make_frame(seed, first_index + i, width, height, num_cells, num_classes, void_class, cls_rgb,
                               cls_depth, rgb + plane * 3 * i, depth_mm + plane * i, labels + plane * i);
            });
        }
        for (auto& th : pool) th.join();
    });
}
