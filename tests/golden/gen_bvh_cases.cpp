// Generates the input sets of the reference's tests/bvh_tests.cpp with the
// same C++ standard-library generators and distributions (std::mt19937,
// std::uniform_real_distribution<float>), so the fixtures reproduce the
// reference test's triangles and rays bit for bit:
//   - 5,000 triangles, seed 42 (topology test, bvh_tests.cpp:91-119)
//   - 2,000 triangles, seed 7, and 2,000 rays, seed 123 (brute-force test,
//     bvh_tests.cpp:121-163)
// Triangle: base ~ U[-10,10]^3, b = base + (s, s, 0), c = base + (0, s, s)
// with s ~ U[0.05, 0.8] drawn in the order of bvh_tests.cpp:80-85. Ray: origin
// = U[-1,1]^3 * 15, direction = normalize(U[-1,1]^3) (bvh_tests.cpp:139-143).
// Constructor arguments are drawn left to right, the order the reference's
// own (clang, macOS) build evaluates `vec3(f(), f(), f())` in.
// Output: raw little-endian float32 files given on the command line.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

static void tris(unsigned seed, size_t n, const char* path) {
    std::mt19937 rng(seed);
    std::uniform_real_distribution<float> pos(-10.0f, 10.0f);
    std::uniform_real_distribution<float> size(0.05f, 0.8f);
    std::vector<float> out;
    for (size_t i = 0; i < n; ++i) {
        const float bx = pos(rng), by = pos(rng), bz = pos(rng);
        const float s0 = size(rng), s1 = size(rng);
        const float s2 = size(rng), s3 = size(rng);
        const float v[9] = {bx, by, bz, bx + s0, by + s1, bz + 0.0f, bx + 0.0f, by + s2, bz + s3};
        out.insert(out.end(), v, v + 9);
    }
    FILE* f = std::fopen(path, "wb");
    std::fwrite(out.data(), 4, out.size(), f);
    std::fclose(f);
}

static void rays(unsigned seed, size_t n, const char* path) {
    std::mt19937 rng(seed);
    std::uniform_real_distribution<float> u(-1.0f, 1.0f);
    std::vector<float> out;
    for (size_t i = 0; i < n; ++i) {
        const float ox = u(rng) * 15.0f, oy = u(rng) * 15.0f, oz = u(rng) * 15.0f;
        float dx = u(rng), dy = u(rng), dz = u(rng);
        float len = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (len < 1e-3f) { dx = 1; dy = 0; dz = 0; len = 1; }
        const float inv = 1.0f / std::sqrt(dx * dx + dy * dy + dz * dz);
        const float v[6] = {ox, oy, oz, dx * inv, dy * inv, dz * inv};
        out.insert(out.end(), v, v + 6);
    }
    FILE* f = std::fopen(path, "wb");
    std::fwrite(out.data(), 4, out.size(), f);
    std::fclose(f);
}

int main(int argc, char** argv) {
    if (argc != 4) return 1;
    tris(42, 5000, argv[1]);
    tris(7, 2000, argv[2]);
    rays(123, 2000, argv[3]);
    return 0;
}
