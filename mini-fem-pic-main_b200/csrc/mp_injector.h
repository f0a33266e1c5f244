// The host injector's state (InjectIons, src/mini-pic.cpp:208-265): the inlet
// faces, the reference's RNG stream and the shared remainder.  Shared by the
// host sampler (mp_host.cpp) and the device sampler (mp_inject.cu).
#pragma once

#include <random>
#include <vector>

struct mp_injector {
    int n_faces = 0;
    std::vector<int> con;       // [n][3]
    std::vector<double> u, v, normal, area, p0;
    std::vector<int> cell;
    std::mt19937 gen;
    std::uniform_real_distribution<double> dist{0, 1.0};
    double rem = 0;
};
