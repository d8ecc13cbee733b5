// Host execution of the batched form's stochastic rounding (csrc/wig_batch.cuh:
// sr_key, sr_word, SrStream, store_round): every value of the input rounded to
// FP32 `steps` times, with the words either of consecutive steps' seeds (mode
// "seeds": the first word of a lane's stream at step s, for the lane whose first
// element is e0 + i) or of one lane's stream (mode "stream": its first `steps`
// words).  Test infrastructure: tests/test_emu_cpu.py checks the results.
//
//   round_emu values_in(double) rounded_out(float, count x steps) steps element0 seeds|stream
#include "shim.h"
#include "wig_batch.cuh"

#include <cstdio>
#include <string>
#include <vector>

int main(int argc, char** argv) {
  if (argc != 6) return 2;
  const bool stream = std::string(argv[5]) == "stream";
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 3;
  std::vector<double> v;
  double x;
  while (std::fread(&x, sizeof x, 1, f) == 1) v.push_back(x);
  std::fclose(f);
  const long steps = std::atol(argv[3]);
  const long long e0 = std::atoll(argv[4]);
  std::vector<float> out;
  out.reserve(v.size() * steps);
  for (size_t i = 0; i < v.size(); ++i) {
    wig::SrStream rs{wig::sr_word(wig::sr_key(0u, 0u), e0 + (long long)i)};
    for (long s = 0; s < steps; ++s) {
      const unsigned u = stream ? rs.next() : wig::SrStream{wig::sr_word(wig::sr_key((unsigned)s, 0u), e0 + (long long)i)}.next();
      out.push_back(wig::store_round(v[i], u));
    }
  }
  FILE* o = std::fopen(argv[2], "wb");
  if (!o) return 4;
  const bool ok = std::fwrite(out.data(), sizeof(float), out.size(), o) == out.size();
  std::fclose(o);
  return ok ? 0 : 4;
}
