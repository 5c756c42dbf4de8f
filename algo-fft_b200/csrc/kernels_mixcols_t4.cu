// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_part_4(std::vector<MixEntry>& v) {
  v.push_back(mix_entry<MixCfg<MixSched<8, 7>, 16, 8, 8>,
                         MixCfg<MixSched<8, 7>, 16, 8, 8>,
                         MixCfg<MixSched<8, 7>, 8, 8, 8>,
                         MixCfg<MixSched<8, 7>, 8, 8, 8>>());  // 56
  v.push_back(mix_entry<MixCfg<MixSched<9, 9>, 16, 7, 0>,
                         MixCfg<MixSched<9, 9>, 16, 7, 0>,
                         MixCfg<MixSched<9, 9>, 8, 7, 0>,
                         MixCfg<MixSched<9, 9>, 8, 7, 0>>());  // 81
  v.push_back(mix_entry<MixCfg<MixSched<14, 8>, 16, 7, 0>,
                         MixCfg<MixSched<14, 8>, 16, 7, 0>,
                         MixCfg<MixSched<14, 8>, 8, 8, 0>,
                         MixCfg<MixSched<14, 8>, 8, 8, 0>>());  // 112
  v.push_back(mix_entry<MixCfg<MixSched<21, 7>, 16, 6, 0>,
                         MixCfg<MixSched<21, 7>, 16, 6, 0>,
                         MixCfg<MixSched<21, 7>, 8, 6, 0>,
                         MixCfg<MixSched<21, 7>, 8, 6, 0>>());  // 147
  v.push_back(mix_entry<MixCfg<MixSched<16, 12>, 16, 3, 16>,
                         MixCfg<MixSched<16, 12>, 16, 3, 16>,
                         MixCfg<MixSched<16, 12>, 8, 4, 0>,
                         MixCfg<MixSched<16, 12>, 8, 4, 0>>());  // 192
  v.push_back(mix_entry<MixCfg<MixSched<27, 9>, 16, 4, 0>,
                         MixCfg<MixSched<27, 9>, 16, 4, 0>,
                         MixCfg<MixSched<27, 9>, 8, 3, 0>,
                         MixCfg<MixSched<27, 9>, 8, 3, 0>>());  // 243
  v.push_back(mix_entry<MixCfg<MixSched<21, 14>, 16, 3, 0>,
                         MixCfg<MixSched<21, 14>, 16, 3, 0>,
                         MixCfg<MixSched<21, 14>, 8, 2, 0>,
                         MixCfg<MixSched<21, 14>, 8, 2, 0>>());  // 294
  v.push_back(mix_entry<MixCfg<MixSched<20, 18>, 16, 2, 20>,
                         MixCfg<MixSched<20, 18>, 16, 2, 20>,
                         MixCfg<MixSched<20, 18>, 8, 2, 20>,
                         MixCfg<MixSched<20, 18>, 8, 2, 20>>());  // 360
  v.push_back(mix_entry<MixCfg<MixSched<24, 18>, 16, 2, 0>,
                         MixCfg<MixSched<24, 18>, 16, 2, 0>,
                         MixCfg<MixSched<24, 18>, 8, 2, 24>,
                         MixCfg<MixSched<24, 18>, 8, 2, 24>>());  // 432
  v.push_back(mix_entry<MixCfg<MixSched<24, 21>, 8, 3, 24>,
                         MixCfg<MixSched<24, 21>, 8, 3, 24>,
                         MixCfg<MixSched<24, 21>, 4, 4, 24>,
                         MixCfg<MixSched<24, 21>, 4, 4, 24>>());  // 504
  v.push_back(mix_entry<MixCfg<MixSched<25, 24>, 8, 3, 25>,
                         MixCfg<MixSched<25, 24>, 8, 3, 25>,
                         MixCfg<MixSched<25, 24>, 4, 3, 25>,
                         MixCfg<MixSched<25, 24>, 4, 3, 25>>());  // 600
  v.push_back(mix_entry<MixCfg<MixSched<28, 25>, 8, 3, 28>,
                         MixCfg<MixSched<28, 25>, 8, 3, 28>,
                         MixCfg<MixSched<28, 25>, 4, 2, 28>,
                         MixCfg<MixSched<28, 25>, 4, 2, 28>>());  // 700
  v.push_back(mix_entry<MixCfg<MixSched<32, 25>, 8, 2, 32>,
                         MixCfg<MixSched<32, 25>, 8, 2, 32>,
                         MixCfg<MixSched<32, 25>, 4, 2, 32>,
                         MixCfg<MixSched<32, 25>, 4, 2, 32>>());  // 800
  v.push_back(mix_entry<MixCfg<MixSched<35, 27>, 8, 2, 35>,
                         MixCfg<MixSched<35, 27>, 8, 2, 35>,
                         MixCfg<MixSched<35, 27>, 4, 1, 0>,
                         MixCfg<MixSched<35, 27>, 4, 1, 0>>());  // 945
}

}  // namespace gfft
