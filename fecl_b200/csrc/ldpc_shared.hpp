// Shared LDPC launches of a mixed batch (batch.cu) or of a server batch (server.cu):
// the LDPC jobs that take the packed FP16 decoder, grouped by check-degree class,
// every class's frame groups packed into waves that fit in L2 and decoded either with
// one launch per pass over all of a wave's groups (h2_check_many / h2_bit_many) or by
// one cooperative launch per class (h2_multi).  Each job keeps its own scratch, stage
// and finish launches; the results are those of decoding each job alone, bit for bit.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "codec.hpp"

namespace fecl {
namespace capi {

struct SharedLdpcJob {
  fecl_codec_s* c = nullptr;
  uint64_t n = 0;
  const void* llr = nullptr;
  int32_t dtype = FECL_F32;
  uint8_t* msg = nullptr;
  int32_t* iters = nullptr;
  size_t scratch_off = 0;  // in the caller's device arena
  fecl::LdpcLanesParams lp;
};

class SharedLdpc {
 public:
  // Whether a job of codec c joins the shared launch: the packed FP16 decoder with
  // the built-in kernel choice.
  static bool eligible(fecl_codec_s* c) { return c->kind == 0 && c->kernel_sel == FECL_KERNEL_AUTO && c->ldpc_h2_ok(); }
  static size_t scratch_bytes(const SharedLdpcJob& j) {
    return fecl::ldpc_lanes_h2_scratch_bytes(int64_t(j.c->parity()), int64_t(j.c->state()), int64_t(j.n));
  }
  // Bytes of the tables of the launches of up to `codes` codes and `groups` groups
  // (an upper bound, for admission).
  static size_t table_bytes_bound(size_t codes, size_t groups) {
    return 4 * 256 * (codes + 3) + codes * sizeof(fecl::LdpcLanesParams) + groups * (sizeof(fecl::LdpcMultiGroup) + 4);
  }

  std::vector<SharedLdpcJob> jobs;

  // Plans the launches over `jobs` and carves their tables out of cv: one pass per
  // check-degree class (split_classes, needed by the persistent form) or one for every
  // class, its groups in waves of at most wave_bytes of working set.
  void plan(Carver& cv, bool split_classes = true, int64_t wave_bytes = kWaveBytes) {
    passes_.clear();
    std::map<int, std::vector<int>> by_class;
    for (size_t i = 0; i < jobs.size(); ++i) {
      const int d = jobs[i].c->ldev.d_max;
      by_class[split_classes ? (d <= 8 ? 8 : (d <= 16 ? 16 : 32)) : 0].push_back(int(i));
    }
    for (auto& kv : by_class) {
      for (size_t j0 = 0; j0 < kv.second.size(); j0 += fecl::kMultiMaxCodes) {
        Pass ml;
        ml.d_max = kv.first;
        ml.wave_ptr.push_back(0);
        int64_t bytes = 0;
        int in_wave = 0;
        for (size_t j = j0; j < kv.second.size() && j < j0 + fecl::kMultiMaxCodes; ++j) {
          const SharedLdpcJob& s = jobs[kv.second[j]];
          ml.jobs.push_back(kv.second[j]);
          const int64_t gb = fecl::ldpc_lanes_h2_group_bytes(s.c->ldev.N, s.c->ldev.E);
          const int groups = int((s.n + 63) / 64);
          for (int g = 0; g < groups; ++g) {
            if (in_wave > 0 && (bytes + gb > wave_bytes || in_wave == fecl::kMultiMaxWaveGroups)) {
              ml.wave_ptr.push_back(int32_t(ml.groups.size()));
              bytes = 0;
              in_wave = 0;
            }
            fecl::LdpcMultiGroup gr;
            gr.code = int32_t(ml.jobs.size() - 1);
            gr.group = g;
            ml.groups.push_back(gr);
            bytes += gb;
            ++in_wave;
          }
        }
        ml.wave_ptr.push_back(int32_t(ml.groups.size()));
        ml.codes_off = cv.take(ml.jobs.size() * sizeof(fecl::LdpcLanesParams));
        ml.groups_off = cv.take(ml.groups.size() * sizeof(fecl::LdpcMultiGroup));
        ml.waves_off = cv.take(ml.wave_ptr.size() * sizeof(int32_t));
        ml.barrier_off = cv.take(2 * sizeof(unsigned));
        passes_.push_back(std::move(ml));
      }
    }
  }

  // Fills every job's decoder parameters over the device arena at dev_base and writes
  // the tables' image at the same offsets from host_base; the caller copies the range
  // [tables_begin(), tables_end()) to the device before the launches run.
  void fill(char* dev_base, char* host_base) {
    for (auto& j : jobs) {
      Launch d;
      d.llr = j.llr;
      d.hard = j.msg;
      d.iters = j.iters;
      j.lp = lanes_params(j.c, d, j.n, j.dtype, FECL_F32);
      fecl::ldpc_lanes_h2_layout(j.lp, dev_base + j.scratch_off);
    }
    for (auto& ml : passes_) {
      auto* codes = reinterpret_cast<fecl::LdpcLanesParams*>(host_base + ml.codes_off);
      for (size_t i = 0; i < ml.jobs.size(); ++i) codes[i] = jobs[ml.jobs[i]].lp;
      std::memcpy(host_base + ml.groups_off, ml.groups.data(), ml.groups.size() * sizeof(fecl::LdpcMultiGroup));
      std::memcpy(host_base + ml.waves_off, ml.wave_ptr.data(), ml.wave_ptr.size() * sizeof(int32_t));
    }
  }

  // Byte range of the tables (offsets from the arena base).
  size_t tables_begin() const {
    size_t b = SIZE_MAX;
    for (auto& ml : passes_) b = std::min(b, ml.codes_off);
    return passes_.empty() ? 0 : b;
  }
  size_t tables_end() const {
    size_t e = 0;
    for (auto& ml : passes_) e = std::max(e, ml.barrier_off + 2 * sizeof(unsigned));
    return e;
  }

  // Stage every job, run every class's passes (persistent: one cooperative launch per
  // class; else one launch per pass over each wave's groups), finish every job, all on
  // stream s.
  void launch(char* dev_base, cudaStream_t s, bool persistent) const {
    for (auto& j : jobs) cuda_check(fecl::launch_ldpc_h2_stage(j.lp, s), "LDPC stage");
    for (auto& ml : passes_) {
      const fecl::LdpcMultiParams m = params(ml, dev_base);
      if (persistent) {
        cuda_check(fecl::launch_ldpc_h2_multi(m, ml.d_max, s), "LDPC shared launch");
        continue;
      }
      for (size_t w = 0; w + 1 < ml.wave_ptr.size(); ++w) {
        fecl::LdpcManyWave wave;
        wave.q0 = ml.wave_ptr[w];
        wave.groups = ml.wave_ptr[w + 1] - ml.wave_ptr[w];
        for (int q = wave.q0; q < wave.q0 + wave.groups; ++q) {
          const fecl::LdpcLanesParams& p = jobs[ml.jobs[ml.groups[q].code]].lp;
          wave.max_rows = std::max(wave.max_rows, p.M);
          wave.max_bits = std::max(wave.max_bits, p.N);
          wave.iterations = std::max(wave.iterations, p.iterations);
        }
        cuda_check(fecl::launch_ldpc_h2_many(m, wave, ml.d_max, s), "LDPC shared passes");
      }
    }
    for (auto& j : jobs) cuda_check(fecl::launch_ldpc_h2_finish(j.lp, s), "LDPC finish");
  }

  // One line per pass.
  std::string describe(bool persistent) const {
    std::string t;
    for (auto& ml : passes_)
      t += std::string(persistent ? "ldpc shared persistent launch" : "ldpc shared launches per pass") +
           (ml.d_max ? " (check degree <= " + std::to_string(ml.d_max) + "): " : " (every check degree): ") +
           std::to_string(ml.jobs.size()) + " codes, " +
           std::to_string(ml.groups.size()) + " groups of 64 frames in " + std::to_string(ml.wave_ptr.size() - 1) +
           " waves\n";
    return t;
  }
  bool empty() const { return passes_.empty(); }

  // Waves hold at most this many bytes of working set (the packed decoder's own cap).
  static constexpr int64_t kWaveBytes = 96ll << 20;

 private:
  struct Pass {
    int d_max = 0;
    std::vector<int> jobs;
    std::vector<fecl::LdpcMultiGroup> groups;
    std::vector<int32_t> wave_ptr;
    size_t codes_off = 0, groups_off = 0, waves_off = 0, barrier_off = 0;
  };
  std::vector<Pass> passes_;

  static fecl::LdpcMultiParams params(const Pass& ml, char* base) {
    fecl::LdpcMultiParams m;
    m.codes = reinterpret_cast<const fecl::LdpcLanesParams*>(base + ml.codes_off);
    m.ncodes = int32_t(ml.jobs.size());
    m.groups = reinterpret_cast<const fecl::LdpcMultiGroup*>(base + ml.groups_off);
    m.wave_ptr = reinterpret_cast<const int32_t*>(base + ml.waves_off);
    m.nwaves = int32_t(ml.wave_ptr.size()) - 1;
    m.barrier = reinterpret_cast<unsigned*>(base + ml.barrier_off);
    return m;
  }
};

}  // namespace capi
}  // namespace fecl
