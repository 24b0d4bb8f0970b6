// A caller written against the reference's managers (main.cu:98-317 call order), built on
// include/anitowave.hpp.  Reads particles from argv[1] (float32 n x 6: pos, vel), grid settings
// from argv[2..], writes the results to argv[1] + ".out" (float32):
//   VELOCITY_X|Y|Z after P2GTransfer::run, particle velocities after performG2P, positions after
//   advect, level-0 x after two runCycle calls, then the level-0 b it solved for.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#define ANITOWAVE_GLOBAL_NAMES
#include "anitowave.hpp"

static void cu(cudaError_t e) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "CUDA: %s\n", cudaGetErrorString(e));
        std::exit(2);
    }
}

int main(int argc, char** argv) {
    if (argc < 8) {
        std::fprintf(stderr, "usage: %s particles.bin D blockSize baseRes levels th0 th1\n", argv[0]);
        return 1;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 1;
    std::fseek(f, 0, SEEK_END);
    const long bytes = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    const uint32_t n = (uint32_t)(bytes / (6 * sizeof(float)));
    std::vector<float> h(6 * (size_t)n);
    if (std::fread(h.data(), sizeof(float), h.size(), f) != h.size()) return 1;
    std::fclose(f);
    const int D = std::atoi(argv[2]);
    const float bs = (float)std::atof(argv[3]);
    const int base = std::atoi(argv[4]), levels = std::atoi(argv[5]);
    const int32_t th[2] = {std::atoi(argv[6]), std::atoi(argv[7])};
    std::vector<float> hp(3 * (size_t)n), hv(3 * (size_t)n);
    for (size_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            hp[3 * i + a] = h[6 * i + a];
            hv[3 * i + a] = h[6 * i + 3 + a];
        }
    float *dp, *dv;
    cu(cudaMalloc(&dp, hp.size() * sizeof(float)));
    cu(cudaMalloc(&dv, hv.size() * sizeof(float)));
    cu(cudaMemcpy(dp, hp.data(), hp.size() * sizeof(float), cudaMemcpyHostToDevice));
    cu(cudaMemcpy(dv, hv.data(), hv.size() * sizeof(float), cudaMemcpyHostToDevice));
    std::vector<float> out;
    try {
        const int dims[3] = {D, D, D};
        const float dmin[3] = {0.f, 0.f, 0.f};
        MSBGManager mg(dims, bs, dmin, base, levels);
        mg.levelsFromParticles(dp, n, th);
        mg.enforceGrading();
        mg.allocateChannels();
        uint32_t tot[4];
        mg.totals(tot);
        P2GTransfer p2g;
        p2g.run(mg, dp, dv, n);
        for (int a = 0; a < 3; ++a) {
            std::vector<float> u(tot[1 + a]);
            cu(cudaMemcpy(u.data(), mg.channel(AW_VELOCITY_X + a), u.size() * sizeof(float), cudaMemcpyDeviceToHost));
            out.insert(out.end(), u.begin(), u.end());
        }
        G2PManager g2p;
        g2p.init(mg);
        g2p.backupGridVelocity(mg);
        g2p.performG2P(mg, dv, dp, n, 0.95f);
        g2p.advect(mg, dp, n, 1.0f / 240);
        cu(cudaMemcpy(hv.data(), dv, hv.size() * sizeof(float), cudaMemcpyDeviceToHost));
        cu(cudaMemcpy(hp.data(), dp, hp.size() * sizeof(float), cudaMemcpyDeviceToHost));
        out.insert(out.end(), hv.begin(), hv.end());
        out.insert(out.end(), hp.begin(), hp.end());
        g2p.cleanup();
        VCycleSolver solver(0, mg.numBlocks());
        solver.init(mg);
        uint32_t nc = 0;
        float* b = solver.levelArray(0, 1, &nc);
        std::vector<float> hb(nc);
        for (uint32_t i = 0; i < nc; ++i) hb[i] = (float)((i * 2654435761u) % 1000u) / 1000.f - 0.5f;
        cu(cudaMemcpy(b, hb.data(), nc * sizeof(float), cudaMemcpyHostToDevice));
        solver.runCycle(mg, 0);
        solver.runCycle(mg, 0);
        std::vector<float> hx(nc);
        cu(cudaMemcpy(hx.data(), solver.levelArray(0, 0), nc * sizeof(float), cudaMemcpyDeviceToHost));
        out.insert(out.end(), hx.begin(), hx.end());
        out.insert(out.end(), hb.begin(), hb.end());
        // errors come back as exceptions with the library's message
        bool threw = false;
        try {
            solver.runCycle(mg, 1);
        } catch (const anitowave::Error& e) {
            threw = e.status == AW_ERR_UNSUPPORTED;
        }
        if (!threw) return 3;
    } catch (const anitowave::Error& e) {
        std::fprintf(stderr, "anitowave error %d: %s\n", (int)e.status, e.what());
        return 4;
    }
    std::string op = std::string(argv[1]) + ".out";
    FILE* g = std::fopen(op.c_str(), "wb");
    std::fwrite(out.data(), sizeof(float), out.size(), g);
    std::fclose(g);
    std::printf("ok %u particles, %zu floats\n", n, out.size());
    return 0;
}
