// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_rows_part_0(std::vector<MixRowsEntry>& v) {
  v.push_back(mix_rows_entry<MixCfg<MixSched<8, 6>, 64, 2, 0>,
                              MixCfg<MixSched<8, 6>, 64, 1, 8>>());  // 48
  v.push_back(mix_rows_entry<MixCfg<MixSched<8, 7>, 64, 2, 8>,
                              MixCfg<MixSched<8, 7>, 64, 1, 8>>());  // 56
  v.push_back(mix_rows_entry<MixCfg<MixSched<10, 7>, 64, 2, 0>,
                              MixCfg<MixSched<10, 7>, 32, 2, 0>>());  // 70
  v.push_back(mix_rows_entry<MixCfg<MixSched<9, 9>, 32, 3, 0>,
                              MixCfg<MixSched<9, 9>, 32, 2, 0>>());  // 81
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 7>, 64, 2, 0>,
                              MixCfg<MixSched<14, 7>, 32, 2, 0>>());  // 98
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 8>, 64, 1, 0>,
                              MixCfg<MixSched<14, 8>, 32, 2, 0>>());  // 112
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 8>, 32, 3, 0>,
                              MixCfg<MixSched<16, 8>, 16, 4, 0>>());  // 128
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 7>, 32, 3, 0>,
                              MixCfg<MixSched<21, 7>, 16, 3, 0>>());  // 147
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 12>, 32, 2, 14>,
                              MixCfg<MixSched<14, 12>, 16, 2, 14>>());  // 168
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 12>, 32, 1, 16>,
                              MixCfg<MixSched<16, 12>, 16, 2, 0>>());  // 192
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 12>, 32, 1, 0>,
                              MixCfg<MixSched<18, 12>, 16, 2, 0>>());  // 216
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 9>, 32, 2, 0>,
                              MixCfg<MixSched<27, 9>, 16, 2, 0>>());  // 243
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 16>, 16, 3, 0>,
                              MixCfg<MixSched<16, 16>, 8, 4, 0>>());  // 256
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 14>, 16, 3, 0>,
                              MixCfg<MixSched<21, 14>, 8, 2, 0>>());  // 294
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 18>, 16, 2, 0>,
                              MixCfg<MixSched<18, 18>, 8, 3, 0>>());  // 324
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 18>, 16, 2, 20>,
                              MixCfg<MixSched<20, 18>, 8, 2, 20>>());  // 360
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 14>, 16, 3, 0>,
                              MixCfg<MixSched<28, 14>, 8, 2, 0>>());  // 392
  v.push_back(mix_rows_entry<MixCfg<MixSched<24, 18>, 16, 2, 0>,
                              MixCfg<MixSched<24, 18>, 8, 2, 24>>());  // 432
  v.push_back(mix_rows_entry<MixCfg<MixSched<24, 20>, 16, 1, 24>,
                              MixCfg<MixSched<24, 20>, 8, 2, 24>>());  // 480
  v.push_back(mix_rows_entry<MixCfg<MixSched<24, 21>, 8, 3, 24>,
                              MixCfg<MixSched<24, 21>, 4, 4, 24>>());  // 504
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 20>, 8, 3, 0>,
                              MixCfg<MixSched<28, 20>, 4, 2, 28>>());  // 560
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 24>, 8, 3, 25>,
                              MixCfg<MixSched<25, 24>, 4, 3, 25>>());  // 600
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 24>, 8, 3, 27>,
                              MixCfg<MixSched<27, 24>, 4, 2, 27>>());  // 648
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 25>, 8, 3, 28>,
                              MixCfg<MixSched<28, 25>, 4, 2, 28>>());  // 700
  v.push_back(mix_rows_entry<MixCfg<MixSched<30, 25>, 8, 2, 30>,
                              MixCfg<MixSched<30, 25>, 4, 2, 30>>());  // 750
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 25>, 8, 2, 32>,
                              MixCfg<MixSched<32, 25>, 4, 2, 32>>());  // 800
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 25>, 8, 2, 35>,
                              MixCfg<MixSched<35, 25>, 4, 1, 0>>());  // 875
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 27>, 8, 2, 35>,
                              MixCfg<MixSched<35, 27>, 4, 1, 0>>());  // 945
  v.push_back(mix_rows_entry<MixCfg<MixSched<40, 25>, 4, 3, 0>,
                              MixCfg<MixSched<40, 25>, 2, 3, 0>>());  // 1000
}

}  // namespace gfft
