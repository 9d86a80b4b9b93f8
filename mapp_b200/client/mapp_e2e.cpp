// A C++ client of the C ABI doing what a MAPP force loop does each step, for
// the end-to-end measurement: new positions and concentrations from host
// memory (update_0 / update(c)), force_calc, forces and energies back to host
// memory.  The system is set up from a CFG file and the force field's own
// ff_coef arguments, as a MAPP input script would (ReadCFG, ff_coef,
// ForceField::init).
//
//   mapp_e2e <style> <cfg file> <steps> <warmup> <device> <skin> <coef arg>...
//
// Prints one JSON line: the device time of the timed steps (CUDA events on the
// library's stream, every host gap included), the bytes copied per step and
// the first site's force components (a check that forces came back).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mapp_b200.h"

namespace {

int check(int rc, const char* what)
{
    if (rc != MG_OK) {
        std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, mg_last_error());
        std::exit(1);
    }
    return rc;
}

void check_cuda(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) {
        std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
        std::exit(1);
    }
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 8) {
        std::fprintf(stderr, "usage: mapp_e2e style cfg steps warmup device skin coef-args...\n");
        return 2;
    }
    const char* style = argv[1];
    const char* cfg_path = argv[2];
    const int steps = std::atoi(argv[3]), warmup = std::atoi(argv[4]), device = std::atoi(argv[5]);
    const double skin = std::atof(argv[6]);
    const int dmd = std::strncmp(style, "DMD", 3) == 0;
    check_cuda(cudaSetDevice(device), "cudaSetDevice");

    // ReadCFG
    mg_cfg* cfg = nullptr;
    check(mg_cfg_read(cfg_path, dmd, &cfg), "mg_cfg_read");
    int natms = 0, nt = 0, has_v = 0;
    double H[9];
    check(mg_cfg_info(cfg, &natms, &nt, H, &has_v), "mg_cfg_info");
    const int name_len = 64;
    std::vector<char> names((size_t)nt * name_len);
    std::vector<double> masses(nt);
    check(mg_cfg_types(cfg, names.data(), name_len, masses.data()), "mg_cfg_types");
    const int x_dim = dmd ? 3 + nt : 3;
    std::vector<double> s_frac((size_t)natms * x_dim), conc(dmd ? (size_t)natms * nt : 1);
    std::vector<int> type(dmd ? 1 : natms);
    check(mg_cfg_atoms(cfg, s_frac.data(), dmd ? nullptr : type.data(), dmd ? conc.data() : nullptr, nullptr),
          "mg_cfg_atoms");
    mg_cfg_free(cfg);

    // the system: types, box, skin, atoms, ff_coef, init
    mg_system* s = nullptr;
    check(mg_create(style, device, &s), "mg_create");
    std::vector<const char*> tn(nt);
    for (int a = 0; a < nt; a++) tn[a] = names.data() + (size_t)a * name_len;
    check(mg_atoms_set_types(s, nt, tn.data(), masses.data()), "mg_atoms_set_types");
    check(mg_atoms_set_box(s, H), "mg_atoms_set_box");
    check(mg_atoms_set_skin(s, skin), "mg_atoms_set_skin");
    check(mg_atoms_set(s, natms, s_frac.data(), dmd ? nullptr : type.data(), dmd ? conc.data() : nullptr),
          "mg_atoms_set");
    std::vector<const char*> args;
    for (int k = 7; k < argc; k++) args.push_back(argv[k]);
    check(mg_ff_coef(s, (int)args.size(), args.data()), "mg_ff_coef");
    check(mg_ff_init(s), "mg_ff_init");
    cudaStream_t st;
    check_cuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
    check(mg_set_stream(s, st), "mg_set_stream");
    // a production caller reads no per-call device times: no timing events
    check(mg_set_timing(s, 0), "mg_set_timing");

    // pinned host buffers, as a caller keeping its arrays page-locked would
    const size_t nx = (size_t)natms * x_dim, nc = dmd ? (size_t)natms * nt : 0;
    double *x = nullptr, *c = nullptr, *f = nullptr;
    check_cuda(cudaMallocHost(&x, nx * sizeof(double)), "cudaMallocHost");
    check_cuda(cudaMallocHost(&f, nx * sizeof(double)), "cudaMallocHost");
    if (dmd) {
        check_cuda(cudaMallocHost(&c, nc * sizeof(double)), "cudaMallocHost");
        std::memcpy(c, conc.data(), nc * sizeof(double));
    }
    check(mg_atoms_get_x(s, x), "mg_atoms_get_x");
    double en[7];
    auto step = [&]() {
        check(mg_atoms_update_x(s, x, nullptr), "mg_atoms_update_x");
        if (dmd) check(mg_atoms_update_c(s, c), "mg_atoms_update_c");
        check(mg_ff_force_calc(s, 1, f, en), "mg_ff_force_calc");
    };
    for (int k = 0; k < warmup; k++) step();
    check_cuda(cudaStreamSynchronize(st), "sync");
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "event");
    check_cuda(cudaEventCreate(&e1), "event");
    check_cuda(cudaEventRecord(e0, st), "event");
    for (int k = 0; k < steps; k++) step();
    check_cuda(cudaEventRecord(e1, st), "event");
    check_cuda(cudaEventSynchronize(e1), "event");
    float ms = 0.0f;
    check_cuda(cudaEventElapsedTime(&ms, e0, e1), "event");
    std::printf("{\"natms\": %d, \"steps\": %d, \"ms\": %.6f, \"h2d_bytes_per_step\": %zu, "
                "\"d2h_bytes_per_step\": %zu, \"energy\": %.12e, \"f0\": [%.12e, %.12e, %.12e]}\n",
                // (down: f, then the library's one copy of 8 totals and 8 status words)
                natms, steps, ms, (nx + nc) * sizeof(double), nx * sizeof(double) + 8 * sizeof(double) + 8 * sizeof(int),
                en[0], f[0],
                f[1], f[2]);
    mg_destroy(s);
    cudaFreeHost(x);
    cudaFreeHost(f);
    if (c) cudaFreeHost(c);
    cudaStreamDestroy(st);
    return 0;
}
