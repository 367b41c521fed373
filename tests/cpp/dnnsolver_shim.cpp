// Drives include/drwc_dnnsolver.hpp the way the reference's walker drives its
// dnnsolver classes: reads n queries (layers n x 30 floats, cuboids n x 105
// floats, axes n int32) from argv[1], writes to argv[2] in this order:
//   Poisson sample (3n floats), Poisson sample with axes (3n, warns once),
//   gradient sample (5n), ParallelSampler Poisson results in submission order
//   (3n, fresh solver), ParallelSampler gradient results (5n, fresh solver),
//   structureConstruction maxima (n floats),
// and exits 0 when the gradient solver without axes and a null sampler both
// threw as the reference classes do.
#include <cstdio>
#include <fstream>
#include <future>
#include <iostream>
#include <vector>

#include "drwc_dnnsolver.hpp"

using namespace drwc_dnnsolver;

int main(int argc, char** argv) {
    if (argc != 3) {
        std::cerr << "usage: dnnsolver_shim QUERIES OUT\n";
        return 2;
    }
    std::ifstream in(argv[1], std::ios::binary);
    int32_t n = 0;
    in.read(reinterpret_cast<char*>(&n), 4);
    std::vector<float> L((size_t)n * kLayerStride), C((size_t)n * kCuboidStride);
    std::vector<int> ax(n);
    in.read(reinterpret_cast<char*>(L.data()), L.size() * 4);
    in.read(reinterpret_cast<char*>(C.data()), C.size() * 4);
    in.read(reinterpret_cast<char*>(ax.data()), ax.size() * 4);
    if (!in) {
        std::cerr << "short query file\n";
        return 2;
    }
    std::vector<float> out;
    auto put = [&](const std::vector<float>& v) { out.insert(out.end(), v.begin(), v.end()); };
    try {
        DNNSolverPoisson p(0);
        p.loadModels(true);
        put(p.sample(L, C));
        put(p.sample(L, C, ax));
        DNNSolverGrad g(0);
        g.loadModels();
        put(g.sample(L, C, ax));
        bool threw = false;
        try {
            g.sample(L, C);
        } catch (const std::runtime_error&) {
            threw = true;
        }
        if (!threw) return 3;
        threw = false;
        try {
            ParallelSampler bad(nullptr, 3, 8);
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        if (!threw) return 4;
        for (int kind = 0; kind < 2; ++kind) {
            DNNSolverPoisson p2(0);
            DNNSolverGrad g2(0);
            ParallelSampler ps(kind == 0 ? (DNNSolver*)&p2 : (DNNSolver*)&g2, kind == 0 ? 3 : 5, 16);
            std::vector<std::future<std::vector<float>>> fs;
            for (int q = 0; q < n; ++q) {
                std::vector<float> l(L.begin() + (size_t)q * kLayerStride,
                                     L.begin() + (size_t)(q + 1) * kLayerStride);
                std::vector<float> c(C.begin() + (size_t)q * kCuboidStride,
                                     C.begin() + (size_t)(q + 1) * kCuboidStride);
                fs.push_back(kind == 0 ? ps.submit(l, c) : ps.submit(l, c, ax[q]));
            }
            for (auto& f : fs) put(f.get());
        }
        put(p.structureConstruction(L, C, n).second);
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 1;
    }
    std::ofstream o(argv[2], std::ios::binary);
    o.write(reinterpret_cast<const char*>(out.data()), out.size() * 4);
    return o ? 0 : 1;
}
