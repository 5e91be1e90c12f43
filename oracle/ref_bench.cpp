// Timing driver for the upstream dip-fmm reference (test / baseline
// infrastructure only; built by oracle/ref.mk into oracle/_ref/).
//
// It builds cdfmm::UniformFmm(sources, targets, options) exactly as a
// reference user would (include/cdfmm/uniform_fmm.hpp:180-182 upstream), runs
// `warmup` untimed and `steps` timed evaluate_into / evaluate_into_float32
// calls (src/uniform_fmm.cpp:1065-1257 and :1281-1457 upstream), and writes
// the last results plus a one-line JSON timing summary.  A timed step
// evaluates every state once.  With the CudaFull backend (the reference's
// own GPU path, src/cuda_fmm.cu:3457-3655 upstream; FP32, field only) the
// summary also gives the median per-evaluation device-kernel, H2D and D2H
// seconds the reference itself records (UniformFmm::last_timings).
//
// Input file (little endian), written by tests/ and bench.py:
//   char[8]  "CDFMMIN1"
//   int32    n_src, n_tgt, order, depth, precision(0=f32,1=f64),
//            output_flags(1=phi,2=H,3=both), n_states, warmup, steps,
//            use_fixed_map, has_root, backend(0=CpuStatic,1=CpuReference,2=CudaFull)
//   float64  root_centre[3], root_half_width
//   float64  sources[n_src][3], targets[n_tgt][3]
//   float64  moments[n_states][n_src][3]
//   int32    identities[n_tgt]                 (user order, -1 = none)
// Output file: float64 results[n_states][n_tgt][4] = (phi, Hx, Hy, Hz),
//   int32 source_permutation[n_src], int32 target_permutation[n_tgt].

#include "cdfmm/uniform_fmm.hpp"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <typename T> void read_into(std::ifstream &in, T *dst, std::size_t n) {
  in.read(reinterpret_cast<char *>(dst), static_cast<std::streamsize>(n * sizeof(T)));
  if (!in) throw std::runtime_error("truncated input file");
}

std::vector<cdfmm::Vec3> to_vec3(const std::vector<double> &flat) {
  std::vector<cdfmm::Vec3> out(flat.size() / 3);
  for (std::size_t i = 0; i < out.size(); ++i)
    out[i] = {flat[3 * i], flat[3 * i + 1], flat[3 * i + 2]};
  return out;
}

} // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: ref_bench <input.bin> <output.bin>\n");
    return 2;
  }
  try {
    std::ifstream in(argv[1], std::ios::binary);
    char magic[8];
    read_into(in, magic, 8);
    if (std::memcmp(magic, "CDFMMIN1", 8) != 0) throw std::runtime_error("bad magic");
    int32_t h[12];
    read_into(in, h, 12);
    const int n_src = h[0], n_tgt = h[1], order = h[2], depth = h[3];
    const int precision = h[4], output_flags = h[5], n_states = h[6];
    const int warmup = h[7], steps = h[8], use_fixed = h[9], has_root = h[10];
    const int backend = h[11];
    double root[4];
    read_into(in, root, 4);
    std::vector<double> src(3 * static_cast<std::size_t>(n_src));
    std::vector<double> tgt(3 * static_cast<std::size_t>(n_tgt));
    std::vector<double> mom(3 * static_cast<std::size_t>(n_src) * n_states);
    std::vector<int32_t> ids(static_cast<std::size_t>(n_tgt));
    read_into(in, src.data(), src.size());
    read_into(in, tgt.data(), tgt.size());
    read_into(in, mom.data(), mom.size());
    read_into(in, ids.data(), ids.size());

    cdfmm::UniformFmmOptions options;
    options.precision = precision == 0 ? cdfmm::StaticPrecision::Float32
                                       : cdfmm::StaticPrecision::Float64;
    options.expansion_order = order;
    options.tree.max_level = depth;
    options.backend = backend == 1   ? cdfmm::ExecutionBackend::CpuReference
                      : backend == 2 ? cdfmm::ExecutionBackend::CudaFull
                                     : cdfmm::ExecutionBackend::CpuStatic;
    if (backend == 1) options.m2l_backend = cdfmm::M2LBackend::Reference;
    if (has_root) {
      options.tree.root_centre = cdfmm::Vec3{root[0], root[1], root[2]};
      options.tree.root_half_width = root[3];
    }
    if (use_fixed) options.fixed_target_source_indices = std::vector<int>(ids.begin(), ids.end());

    const auto t0 = std::chrono::steady_clock::now();
    cdfmm::UniformFmm fmm(to_vec3(src), to_vec3(tgt), options);
    const double setup_s =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    const auto flags = static_cast<cdfmm::OutputFlags>(output_flags);
    std::vector<cdfmm::PotentialField> out64(static_cast<std::size_t>(n_tgt));
    std::vector<cdfmm::FloatPotentialField> out32(static_cast<std::size_t>(n_tgt));
    std::vector<double> results(static_cast<std::size_t>(n_states) * n_tgt * 4);
    std::vector<std::vector<cdfmm::Vec3>> states(static_cast<std::size_t>(n_states));
    for (int k = 0; k < n_states; ++k) {
      std::vector<double> part(mom.begin() + static_cast<std::ptrdiff_t>(k) * 3 * n_src,
                               mom.begin() + static_cast<std::ptrdiff_t>(k + 1) * 3 * n_src);
      states[k] = to_vec3(part);
    }
    const std::span<const int> id_span(ids.data(), ids.size());
    auto run_state = [&](int k) {
      if (precision == 0) {
        fmm.evaluate_into_float32(states[k], out32, flags, id_span);
      } else {
        fmm.evaluate_into(states[k], out64, flags, id_span);
      }
    };
    auto store_state = [&](int k) {
      for (int i = 0; i < n_tgt; ++i) {
        double *r = &results[(static_cast<std::size_t>(k) * n_tgt + i) * 4];
        if (precision == 0) {
          r[0] = out32[i].phi; r[1] = out32[i].H.x; r[2] = out32[i].H.y; r[3] = out32[i].H.z;
        } else {
          r[0] = out64[i].phi; r[1] = out64[i].H.x; r[2] = out64[i].H.y; r[3] = out64[i].H.z;
        }
      }
    };
    for (int w = 0; w < warmup; ++w) run_state(w % n_states);
    std::vector<double> step_s, kernel_s, h2d_s, d2h_s;
    for (int s = 0; s < steps; ++s) {
      const auto a = std::chrono::steady_clock::now();
      for (int k = 0; k < n_states; ++k) {
        run_state(k);
        if (backend == 2) {
          const cdfmm::EvaluationTimings &t = fmm.last_timings();
          kernel_s.push_back(t.cuda_kernel.total_seconds);
          h2d_s.push_back(t.cuda_h2d.total_seconds);
          d2h_s.push_back(t.cuda_d2h.total_seconds);
        }
      }
      step_s.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count());
    }
    auto median_of = [](std::vector<double> v) {
      std::sort(v.begin(), v.end());
      return v.empty() ? 0.0 : v[v.size() / 2];
    };
    for (int k = 0; k < n_states; ++k) {
      run_state(k);
      store_state(k);
    }
    std::ofstream out(argv[2], std::ios::binary);
    out.write(reinterpret_cast<const char *>(results.data()),
              static_cast<std::streamsize>(results.size() * sizeof(double)));
    const auto sp = fmm.tree().source_permutation();
    const auto tp = fmm.tree().target_permutation();
    out.write(reinterpret_cast<const char *>(sp.data()), static_cast<std::streamsize>(sp.size() * 4));
    out.write(reinterpret_cast<const char *>(tp.data()), static_cast<std::streamsize>(tp.size() * 4));

    std::vector<double> sorted = step_s;
    std::sort(sorted.begin(), sorted.end());
    const double median = sorted.empty() ? 0.0 : sorted[sorted.size() / 2];
    double total = 0.0;
    for (double v : step_s) total += v;
    int threads = 1;
#ifdef _OPENMP
    threads = omp_get_max_threads();
#endif
    std::printf("{\"setup_s\": %.6f, \"steps\": %d, \"states_per_step\": %d, "
                "\"median_step_s\": %.6f, \"total_timed_s\": %.6f, \"threads\": %d, "
                "\"m2l_classes\": %zu, \"m2l_interactions\": %zu, \"backend\": %d, "
                "\"median_kernel_s\": %.6f, \"median_h2d_s\": %.6f, \"median_d2h_s\": %.6f}\n",
                setup_s, steps, n_states, median, total, threads,
                fmm.static_plan_statistics().transfer_classes,
                fmm.static_plan_statistics().interactions, backend, median_of(kernel_s), median_of(h2d_s),
                median_of(d2h_s));
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "ref_bench error: %s\n", e.what());
    return 1;
  }
}
