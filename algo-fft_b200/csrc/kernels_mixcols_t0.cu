// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_part_0(std::vector<MixEntry>& v) {
  v.push_back(mix_entry<MixCfg<MixSched<8, 6>, 16, 8, 0>,
                         MixCfg<MixSched<8, 6>, 16, 8, 0>,
                         MixCfg<MixSched<8, 6>, 8, 8, 8>,
                         MixCfg<MixSched<8, 6>, 8, 8, 8>>());  // 48
  v.push_back(mix_entry<MixCfg<MixSched<10, 7>, 16, 7, 0>,
                         MixCfg<MixSched<10, 7>, 16, 7, 0>,
                         MixCfg<MixSched<10, 7>, 8, 8, 0>,
                         MixCfg<MixSched<10, 7>, 8, 8, 0>>());  // 70
  v.push_back(mix_entry<MixCfg<MixSched<14, 7>, 16, 7, 0>,
                         MixCfg<MixSched<14, 7>, 16, 7, 0>,
                         MixCfg<MixSched<14, 7>, 8, 8, 0>,
                         MixCfg<MixSched<14, 7>, 8, 8, 0>>());  // 98
  v.push_back(mix_entry<MixCfg<MixSched<16, 8>, 16, 7, 0>,
                         MixCfg<MixSched<16, 8>, 16, 7, 0>,
                         MixCfg<MixSched<16, 8>, 8, 8, 0>,
                         MixCfg<MixSched<16, 8>, 8, 8, 0>>());  // 128
  v.push_back(mix_entry<MixCfg<MixSched<14, 12>, 16, 4, 14>,
                         MixCfg<MixSched<14, 12>, 16, 4, 14>,
                         MixCfg<MixSched<14, 12>, 8, 4, 14>,
                         MixCfg<MixSched<14, 12>, 8, 4, 14>>());  // 168
  v.push_back(mix_entry<MixCfg<MixSched<18, 12>, 16, 3, 0>,
                         MixCfg<MixSched<18, 12>, 16, 3, 0>,
                         MixCfg<MixSched<18, 12>, 8, 4, 0>,
                         MixCfg<MixSched<18, 12>, 8, 4, 0>>());  // 216
  v.push_back(mix_entry<MixCfg<MixSched<16, 16>, 16, 3, 0>,
                         MixCfg<MixSched<16, 16>, 16, 3, 0>,
                         MixCfg<MixSched<16, 16>, 8, 4, 0>,
                         MixCfg<MixSched<16, 16>, 8, 4, 0>>());  // 256
  v.push_back(mix_entry<MixCfg<MixSched<18, 18>, 16, 2, 0>,
                         MixCfg<MixSched<18, 18>, 16, 2, 0>,
                         MixCfg<MixSched<18, 18>, 8, 3, 0>,
                         MixCfg<MixSched<18, 18>, 8, 3, 0>>());  // 324
  v.push_back(mix_entry<MixCfg<MixSched<28, 14>, 16, 3, 0>,
                         MixCfg<MixSched<28, 14>, 16, 3, 0>,
                         MixCfg<MixSched<28, 14>, 8, 2, 0>,
                         MixCfg<MixSched<28, 14>, 8, 2, 0>>());  // 392
  v.push_back(mix_entry<MixCfg<MixSched<10, 8, 6>, 8, 3, 0>,
                         MixCfg<MixSched<10, 8, 6>, 8, 4, 0>,
                         MixCfg<MixSched<24, 20>, 8, 2, 24>,
                         MixCfg<MixSched<24, 20>, 8, 2, 24>>());  // 480
  v.push_back(mix_entry<MixCfg<MixSched<28, 20>, 8, 3, 0>,
                         MixCfg<MixSched<28, 20>, 8, 3, 0>,
                         MixCfg<MixSched<28, 20>, 4, 2, 28>,
                         MixCfg<MixSched<28, 20>, 4, 2, 28>>());  // 560
  v.push_back(mix_entry<MixCfg<MixSched<27, 24>, 8, 3, 27>,
                         MixCfg<MixSched<27, 24>, 8, 3, 27>,
                         MixCfg<MixSched<27, 24>, 4, 2, 27>,
                         MixCfg<MixSched<27, 24>, 4, 2, 27>>());  // 648
  v.push_back(mix_entry<MixCfg<MixSched<30, 25>, 8, 2, 30>,
                         MixCfg<MixSched<30, 25>, 8, 2, 30>,
                         MixCfg<MixSched<30, 25>, 4, 2, 30>,
                         MixCfg<MixSched<30, 25>, 4, 2, 30>>());  // 750
  v.push_back(mix_entry<MixCfg<MixSched<35, 25>, 8, 2, 35>,
                         MixCfg<MixSched<35, 25>, 8, 2, 35>,
                         MixCfg<MixSched<35, 25>, 4, 1, 0>,
                         MixCfg<MixSched<35, 25>, 4, 1, 0>>());  // 875
  v.push_back(mix_entry<MixCfg<MixSched<40, 25>, 8, 2, 0>,
                         MixCfg<MixSched<40, 25>, 8, 2, 0>,
                         MixCfg<MixSched<40, 25>, 4, 1, 0>,
                         MixCfg<MixSched<10, 10, 10>, 4, 2, 0>>());  // 1000
}

}  // namespace gfft
