// The drop-in programs cmf_walk_f64, cmf_walk_df64 and cmf_walk_rns: the
// reference's command lines (README.md:93-106; cmf_walk_f64.cu:318-357,
// cmf_walk_df64.cu:443-462, cmf_walk_rns.cu:414-434) and JSON files
// (cmf_walk_f64.cu:262-305, cmf_walk_df64.cu:425-436,
// cmf_walk_rns.cu:396-407), over the C ABI in include/cmfw.h.
//
// Built three times with CMFW_CLI_VARIANT = 0 (f64), 1 (df64), 2 (rns).
//
// Extensions beyond the reference's flags:
//   --df64-compat     (df64) the reference's float-reciprocal arithmetic
//   --unfused-column  (rns)  round the column polynomial like a CPU build
//   --inputs FILE     raw 192-byte trajectory records instead of the
//                     built-in generators (n_traj = file size / 192)
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "cmfw.h"

#ifndef CMFW_CLI_VARIANT
#define CMFW_CLI_VARIANT 0
#endif

namespace {

const char *kVariantName[3] = {"f64", "df64", "rns"};

void json_double(char *buf, size_t size, double x) {
    if (!std::isfinite(x)) snprintf(buf, size, "null");
    else snprintf(buf, size, "%.17g", x);
}

bool parse_cmf_type(const char *s, int &p, int &q) { return sscanf(s, "%dF%d", &p, &q) == 2; }

}  // namespace

int main(int argc, char **argv) {
    const int variant = CMFW_CLI_VARIANT;
    int p = 6, q = 5;
    double z = 0.5;
    int N = 1000, h = 50, n_traj = 10000, mode = 0;
    int block_size = (variant == 2) ? 128 : 256;
    int n_primes = 8;
    bool use_zeta = false;
    int flags = 0;
    std::string inputs_path;
    std::string output_path = std::string("results_") + kVariantName[variant] + ".json";

    for (int i = 1; i < argc; ++i) {
        std::string arg = argv[i];
        auto next = [&]() -> const char * {
            if (++i >= argc) {
                if (variant == 0) fprintf(stderr, "Missing value after %s\n", argv[i - 1]);
                exit(1);
            }
            return argv[i];
        };
        if (arg == "--cmf" && i + 1 < argc) {
            if (!parse_cmf_type(argv[++i], p, q)) {
                if (variant == 0) fprintf(stderr, "Invalid CMF type: %s (use e.g. 6F5)\n", argv[i]);
                return 1;
            }
        } else if (arg == "--z") z = atof(next());
        else if (arg == "--N") N = atoi(next());
        else if (arg == "--h") h = atoi(next());
        else if (arg == "--n-traj") n_traj = atoi(next());
        else if (arg == "--mode") mode = (strcmp(next(), "delta") == 0) ? 1 : 0;
        else if (arg == "--block-size") block_size = atoi(next());
        else if (arg == "--output") output_path = next();
        else if (arg == "--zeta") { use_zeta = true; z = 1.0; }
        else if (arg == "--n-primes" && variant == 2) n_primes = atoi(next());
        else if (arg == "--df64-compat" && variant == 1) flags |= CMFW_F_DF64_COMPAT;
        else if (arg == "--unfused-column" && variant == 2) flags |= CMFW_F_UNFUSED_COLUMN;
        else if (arg == "--inputs") inputs_path = next();
        else {
            if (variant == 0) fprintf(stderr, "Unknown arg: %s\n", argv[i]);
            else fprintf(stderr, "Unknown: %s\n", argv[i]);
            return 1;
        }
    }

    char banner[512];
    if (cmfw_device_banner(banner, sizeof(banner)) != CMFW_OK) {
        fprintf(stderr, "error: %s\n", cmfw_last_error());
        return 2;
    }
    fprintf(stderr, "%s\n", banner);

    cmfw_desc desc = cmfw_make_desc(p, q, z);
    if (cmfw_check_desc(&desc) != CMFW_OK) {
        fprintf(stderr, "error: %s\n", cmfw_last_error());
        return 1;
    }
    const char *zeta_tag = use_zeta ? " [ZETA]" : "";
    if (variant == 0)
        fprintf(stderr, "=== f64 Benchmark: %dF%d z=%.4f N=%d h=%d n_traj=%d rank=%d%s ===\n", p, q, z, N, h,
                n_traj, desc.rank, zeta_tag);
    else if (variant == 1)
        fprintf(stderr, "=== df64: %dF%d z=%.4f N=%d h=%d n_traj=%d rank=%d%s ===\n", p, q, z, N, h, n_traj,
                desc.rank, zeta_tag);
    else
        fprintf(stderr, "=== RNS: %dF%d z=%.4f N=%d h=%d n_traj=%d rank=%d primes=%d%s ===\n", p, q, z, N, h,
                n_traj, desc.rank, n_primes, zeta_tag);

    std::vector<cmfw_traj_in> in;
    if (!inputs_path.empty()) {
        std::ifstream f(inputs_path, std::ios::binary | std::ios::ate);
        if (!f) { fprintf(stderr, "error: cannot read %s\n", inputs_path.c_str()); return 1; }
        const std::streamsize bytes = f.tellg();
        if (bytes % (std::streamsize)sizeof(cmfw_traj_in) != 0) {
            fprintf(stderr, "error: %s is not a whole number of 192-byte records\n", inputs_path.c_str());
            return 1;
        }
        n_traj = (int)(bytes / (std::streamsize)sizeof(cmfw_traj_in));
        in.resize((size_t)n_traj);
        f.seekg(0);
        f.read(reinterpret_cast<char *>(in.data()), bytes);
    } else {
        if (n_traj < 0) { fprintf(stderr, "error: --n-traj must not be negative\n"); return 1; }
        in.resize((size_t)n_traj);
        if (cmfw_reference_inputs(p, q, n_traj, mode, use_zeta ? 1 : 0, in.data()) != CMFW_OK) {
            fprintf(stderr, "error: %s\n", cmfw_last_error());
            return 1;
        }
    }
    std::vector<cmfw_traj_out> out((size_t)n_traj);
    cmfw_launch L;
    memset(&L, 0, sizeof(L));
    L.block_size = block_size;
    L.flags = flags;
    const cmfw_variant cv = (cmfw_variant)variant;

    // Warm-up on one trajectory, as the reference does before timing.
    if (n_traj > 0) {
        cmfw_traj_out w;
        if (cmfw_walk_host(cv, &desc, in.data(), &w, 1, N, h, n_primes, &L, nullptr, nullptr) != CMFW_OK) {
            fprintf(stderr, "error: %s\n", cmfw_last_error());
            return 2;
        }
    }
    float ms = 0.f;
    if (cmfw_walk_host(cv, &desc, in.data(), out.data(), n_traj, N, h, n_primes, &L, &ms, nullptr) != CMFW_OK) {
        fprintf(stderr, "error: %s\n", cmfw_last_error());
        return 2;
    }
    size_t mem_free = 0, mem_total = 0;
    // Device-wide, like the reference (cmf_walk_f64.cu:236-238).
    cmfw_device_meminfo(&mem_free, &mem_total);
    const double mem_used = (double)(mem_total - mem_free);

    int n_valid = 0, n_with_limits = 0;
    double sum_delta = 0.0;
    for (int i = 0; i < n_traj; ++i) {
        if (out[i].valid) {
            ++n_valid;
            if (!std::isnan(out[i].limit)) ++n_with_limits;
            if (!std::isnan(out[i].delta)) sum_delta += out[i].delta;
        }
    }
    const double avg_delta = n_valid > 0 ? sum_delta / n_valid : NAN;
    const double tps = n_traj / (ms / 1000.0);

    std::ofstream o(output_path);
    if (variant == 0) {
        fprintf(stderr, "  Valid: %d/%d  With limits: %d  Avg delta: %.6f\n", n_valid, n_traj, n_with_limits,
                avg_delta);
        fprintf(stderr, "  GPU time: %.3f ms  Throughput: %.0f traj/s  Mem used: %.2f MB\n", ms, tps,
                mem_used / 1e6);
        o << "{\n";
        o << "  \"variant\": \"f64\",\n";
        o << "  \"cmf\": \"" << p << "F" << q << "\",\n";
        o << "  \"p\": " << p << ", \"q\": " << q << ",\n";
        o << "  \"z\": " << z << ",\n";
        o << "  \"rank\": " << desc.rank << ",\n";
        o << "  \"naxes\": " << desc.naxes << ",\n";
        o << "  \"N\": " << N << ",\n";
        o << "  \"h\": " << h << ",\n";
        o << "  \"n_traj\": " << n_traj << ",\n";
        o << "  \"mode\": \"" << (mode == 0 ? "limit" : "delta") << "\",\n";
        o << "  \"block_size\": " << block_size << ",\n";
        o << "  \"gpu_time_ms\": " << ms << ",\n";
        o << "  \"throughput_traj_per_s\": " << tps << ",\n";
        o << "  \"mem_used_mb\": " << mem_used / 1e6 << ",\n";
        o << "  \"n_valid\": " << n_valid << ",\n";
        o << "  \"n_with_limits\": " << n_with_limits << ",\n";
        o << "  \"avg_delta\": " << (std::isfinite(avg_delta) ? std::to_string(avg_delta) : "null") << ",\n";
        o << "  \"results\": [\n";
        const int shown = n_traj < 100 ? n_traj : 100;
        for (int i = 0; i < shown; ++i) {
            char lb[32], db[32], pb[32], qb[32], prb[32], lsb[32];
            json_double(lb, sizeof(lb), out[i].limit);
            json_double(db, sizeof(db), out[i].delta);
            json_double(pb, sizeof(pb), out[i].p);
            json_double(qb, sizeof(qb), out[i].q);
            json_double(prb, sizeof(prb), out[i].precision);
            json_double(lsb, sizeof(lsb), out[i].log_scale);
            o << "    {\"idx\": " << i << ", \"valid\": " << out[i].valid << ", \"limit\": " << lb
              << ", \"delta\": " << db << ", \"p\": " << pb << ", \"q\": " << qb << ", \"precision\": " << prb
              << ", \"log_scale\": " << lsb << ", \"n_limits\": " << out[i].n_limits << "}";
            if (i < shown - 1) o << ",";
            o << "\n";
        }
        o << "  ]\n";
        o << "}\n";
        fprintf(stderr, "  Results written to: %s\n", output_path.c_str());
    } else {
        fprintf(stderr, "  Valid: %d/%d  Limits: %d  Avg delta: %.6f  Time: %.3f ms  %.0f traj/s  Mem: %.2f MB\n",
                n_valid, n_traj, n_with_limits, avg_delta, ms, tps, mem_used / 1e6);
        o << "{\n  \"variant\": \"" << kVariantName[variant] << "\",\n  \"cmf\": \"" << p << "F" << q << "\",\n";
        o << "  \"p\": " << p << ", \"q\": " << q << ", \"z\": " << z << ",\n";
        o << "  \"rank\": " << desc.rank << ", \"naxes\": " << desc.naxes << ",\n";
        o << "  \"N\": " << N << ", \"h\": " << h << ", \"n_traj\": " << n_traj << ",\n";
        o << "  \"mode\": \"" << (mode == 0 ? "limit" : "delta") << "\",\n";
        if (variant == 2) o << "  \"block_size\": " << block_size << ", \"n_primes\": " << n_primes << ",\n";
        else o << "  \"block_size\": " << block_size << ",\n";
        o << "  \"gpu_time_ms\": " << ms << ", \"throughput_traj_per_s\": " << tps << ",\n";
        o << "  \"mem_used_mb\": " << mem_used / 1e6 << ",\n";
        char dbuf[32];
        json_double(dbuf, sizeof(dbuf), avg_delta);
        o << "  \"n_valid\": " << n_valid << ", \"n_with_limits\": " << n_with_limits << ", \"avg_delta\": " << dbuf
          << "\n}\n";
    }
    return 0;
}
