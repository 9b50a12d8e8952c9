// `wos` command line: the reference launcher's interface (src/main.cpp:22-393)
// over libwos_b200's equation registry.
//
//   wos [options] [equation] [Nx Ny] [Nz] [mesh.obj]
//
// Same options, defaults, validation messages, overwrite protection and exit
// codes as the reference (help 0, errors 1).  Two additions select the GPU
// path: --method plain|fast|fast64 (default plain, the reference's FP64
// estimator and streams) and --device N.
#include <cerrno>
#include <charconv>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <string>
#include <system_error>
#include <vector>

#include "../../include/wos_b200.h"

namespace {

void usage(const char *prog) {
    std::printf(
        "Usage: %s [options] [equation] [Nx Ny] [Nz] [mesh.obj]\n"
        "\n"
        "Options:\n"
        "  -o, --output FILE  HDF5 output path (default: wos.h5)\n"
        "      --seed UINT64  fixed random seed (default: generated from current time)\n"
        "      --walks N      WoS paths per inside grid point (default: 10000)\n"
        "      --epsilon X    boundary stopping distance (default: 0.01)\n"
        "      --max-steps N  maximum steps per WoS path (default: 1000)\n"
        "      --max-ray-attempts N\n"
        "                     maximum 3D inside-test ray attempts (default: 12)\n"
        "      --alpha X      screened Poisson coefficient (default: 5;\n"
        "                     screened_poisson only)\n"
        "      --source-mode MODE\n"
        "                     Poisson source sampling: uniform or green\n"
        "                     (poisson and screened_poisson)\n"
        "      --force        allow an existing output file to be overwritten\n"
        "      --method M     GPU walk method: plain (FP64, reference streams; default),\n"
        "                     fast (FP32 with FP64 epsilon shell) or fast64\n"
        "      --device N     CUDA device (default: 0)\n"
        "  -h, --help         show this help message\n",
        prog);
}

bool parse_int(const char *text, int minimum, int *value) {
    int v = 0;
    const char *end = text + std::strlen(text);
    const auto r = std::from_chars(text, end, v);
    if (r.ec != std::errc{} || r.ptr != end || v < minimum) return false;
    *value = v;
    return true;
}

bool parse_u64(const char *text, uint64_t *value) {
    uint64_t v = 0;
    const char *end = text + std::strlen(text);
    const auto r = std::from_chars(text, end, v);
    if (r.ec != std::errc{} || r.ptr != end) return false;
    *value = v;
    return true;
}

bool parse_positive(const char *text, double *value) {
    if (*text == '\0' || std::isspace(static_cast<unsigned char>(*text))) return false;
    char *end = nullptr;
    errno = 0;
    const double v = std::strtod(text, &end);
    if (end == text || *end != '\0' || errno == ERANGE || !std::isfinite(v) || v <= 0.0) return false;
    *value = v;
    return true;
}

}  // namespace

int main(int argc, char **argv) {
    const char *eq_name = "laplace";
    const char *mesh = "meshes/annulus.obj";
    const char *output = "wos.h5";
    int Nx = 32, Ny = 32, Nz = 32;
    int walks = 10000;
    double epsilon = 1e-2;
    int max_steps = 1000;
    int rays = 12;
    double alpha = 5.0;
    int source_mode = WOS_SOURCE_UNIFORM;
    bool force = false;
    uint64_t seed = 0;
    bool have_seed = false, have_alpha = false, have_mode = false;
    std::vector<const char *> pos;

    // value-taking options: name, what a missing value needs
    auto need = [&](int &i, const char *what) -> const char * {
        if (++i >= argc) {
            std::fprintf(stderr, "%s requires %s\n", argv[i - 1], what);
            return nullptr;
        }
        return argv[i];
    };
    for (int i = 1; i < argc; ++i) {
        const char *a = argv[i];
        if (!std::strcmp(a, "-h") || !std::strcmp(a, "--help")) {
            usage(argv[0]);
            return 0;
        } else if (!std::strcmp(a, "-o") || !std::strcmp(a, "--output")) {
            const char *v = need(i, "a file path");
            if (!v) return 1;
            output = v;
        } else if (!std::strcmp(a, "--seed")) {
            const char *v = need(i, "an unsigned 64-bit integer");
            if (!v) return 1;
            if (!parse_u64(v, &seed)) {
                std::fprintf(stderr, "Invalid --seed value: %s\n", v);
                return 1;
            }
            have_seed = true;
        } else if (!std::strcmp(a, "--walks")) {
            const char *v = need(i, "a positive integer");
            if (!v) return 1;
            if (!parse_int(v, 1, &walks)) {
                std::fprintf(stderr, "Invalid --walks value: %s\n", v);
                return 1;
            }
        } else if (!std::strcmp(a, "--epsilon")) {
            const char *v = need(i, "a positive finite number");
            if (!v) return 1;
            if (!parse_positive(v, &epsilon)) {
                std::fprintf(stderr, "Invalid --epsilon value: %s\n", v);
                return 1;
            }
        } else if (!std::strcmp(a, "--max-steps")) {
            const char *v = need(i, "a positive integer");
            if (!v) return 1;
            if (!parse_int(v, 1, &max_steps)) {
                std::fprintf(stderr, "Invalid --max-steps value: %s\n", v);
                return 1;
            }
        } else if (!std::strcmp(a, "--max-ray-attempts")) {
            const char *v = need(i, "an integer of at least 3");
            if (!v) return 1;
            if (!parse_int(v, 3, &rays)) {
                std::fprintf(stderr, "Invalid --max-ray-attempts value: %s\n", v);
                return 1;
            }
        } else if (!std::strcmp(a, "--alpha")) {
            const char *v = need(i, "a positive finite number");
            if (!v) return 1;
            if (!parse_positive(v, &alpha)) {
                std::fprintf(stderr, "Invalid --alpha value: %s\n", v);
                return 1;
            }
            have_alpha = true;
        } else if (!std::strcmp(a, "--source-mode")) {
            const char *v = need(i, "uniform or green");
            if (!v) return 1;
            if (!std::strcmp(v, "uniform")) {
                source_mode = WOS_SOURCE_UNIFORM;
            } else if (!std::strcmp(v, "green")) {
                source_mode = WOS_SOURCE_GREEN;
            } else {
                std::fprintf(stderr, "Invalid --source-mode value: %s\n", v);
                return 1;
            }
            have_mode = true;
        } else if (!std::strcmp(a, "--method")) {
            const char *v = need(i, "plain, fast or fast64");
            if (!v) return 1;
            if (std::strcmp(v, "plain") && std::strcmp(v, "fast") && std::strcmp(v, "fast64")) {
                std::fprintf(stderr, "Invalid --method value: %s\n", v);
                return 1;
            }
            setenv("WOS_B200_METHOD", v, 1);
        } else if (!std::strcmp(a, "--device")) {
            const char *v = need(i, "a device index");
            if (!v) return 1;
            int d = 0;
            if (!parse_int(v, 0, &d)) {
                std::fprintf(stderr, "Invalid --device value: %s\n", v);
                return 1;
            }
            setenv("WOS_B200_DEVICE", v, 1);
        } else if (!std::strcmp(a, "--force")) {
            force = true;
        } else if (a[0] == '-') {
            std::fprintf(stderr, "Unknown option: %s\n", a);
            return 1;
        } else {
            pos.push_back(a);
        }
    }
    if (pos.size() > 5) {
        std::fprintf(stderr, "Too many positional arguments\n");
        return 1;
    }
    if (pos.size() == 2) {
        std::fprintf(stderr, "Nx and Ny must be provided together\n");
        return 1;
    }
    if (!pos.empty()) eq_name = pos[0];
    if (pos.size() >= 3 && (!parse_int(pos[1], 1, &Nx) || !parse_int(pos[2], 1, &Ny))) {
        std::fprintf(stderr, "Nx and Ny must be positive integers\n");
        return 1;
    }
    if (pos.size() >= 4) {
        int nz = 0;
        if (parse_int(pos[3], 1, &nz)) {
            Nz = nz;
            if (pos.size() == 5) mesh = pos[4];
        } else if (pos.size() == 5) {
            std::fprintf(stderr,
                         "Nz must be a positive integer when a fifth positional argument is present\n");
            return 1;
        } else {
            mesh = pos[3];
        }
    }
    if (!have_seed) {
        seed = static_cast<uint64_t>(std::chrono::high_resolution_clock::now().time_since_epoch().count());
    }
    std::printf("Random seed: %llu%s\n", static_cast<unsigned long long>(seed),
                have_seed ? " (fixed by --seed)" : " (generated from current time)");

    int n_eq = 0;
    const wos_equation_entry *reg = wos_equation_registry(&n_eq);
    const wos_equation_entry *eq = nullptr;
    for (int i = 0; i < n_eq; ++i) {
        if (!std::strcmp(reg[i].name, eq_name)) eq = &reg[i];
    }
    if (!eq) {
        std::fprintf(stderr, "Unknown equation: '%s'\nAvailable equations:\n", eq_name);
        for (int i = 0; i < n_eq; ++i) std::fprintf(stderr, "  - %s\n", reg[i].name);
        return 1;
    }
    if (have_alpha && std::strcmp(eq->name, "screened_poisson")) {
        std::fprintf(stderr,
                     "Warning: --alpha applies only to screened_poisson; it will be ignored for "
                     "equation '%s'.\n",
                     eq->name);
    }
    if (have_mode && std::strcmp(eq->name, "poisson") && std::strcmp(eq->name, "screened_poisson")) {
        std::fprintf(stderr,
                     "Warning: --source-mode applies only to poisson and screened_poisson; it "
                     "will be ignored for equation '%s'.\n",
                     eq->name);
    }
    if (!force) {
        std::error_code ec;
        const bool exists = std::filesystem::exists(output, ec);
        if (ec) {
            std::fprintf(stderr, "Could not inspect output path %s: %s\n", output, ec.message().c_str());
            return 1;
        }
        if (exists) {
            std::fprintf(stderr,
                         "Refusing to overwrite existing output: %s\n"
                         "Choose another path with --output, or pass --force.\n",
                         output);
            return 1;
        }
    }
    const int dim = wos_peek_mesh_dim(mesh);
    if (dim == 0) return 1;
    const wos_run_fn fn = dim == 2 ? eq->run_2D : eq->run_3D;
    return fn(0, 1, mesh, output, Nx, Ny, Nz, walks, epsilon, max_steps, rays, seed, alpha,
              source_mode);
}
