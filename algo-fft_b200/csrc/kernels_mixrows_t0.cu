// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_rows_part_0(std::vector<MixRowsEntry>& v) {
  v.push_back(mix_rows_entry<MixCfg<MixSched<8, 6>, 64, 2, 0>,
                              MixCfg<MixSched<8, 6>, 64, 1, 8>>());  // 48
  v.push_back(mix_rows_entry<MixCfg<MixSched<10, 7>, 64, 2, 0>,
                              MixCfg<MixSched<10, 7>, 32, 2, 0>>());  // 70
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 7>, 64, 2, 0>,
                              MixCfg<MixSched<14, 7>, 32, 2, 0>>());  // 98
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 8>, 32, 3, 0>,
                              MixCfg<MixSched<16, 8>, 16, 4, 0>>());  // 128
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 12>, 32, 2, 14>,
                              MixCfg<MixSched<14, 12>, 16, 2, 14>>());  // 168
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 12>, 32, 1, 0>,
                              MixCfg<MixSched<18, 12>, 16, 2, 0>>());  // 216
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 16>, 16, 3, 0>,
                              MixCfg<MixSched<16, 16>, 8, 4, 0>>());  // 256
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 18>, 16, 2, 0>,
                              MixCfg<MixSched<18, 18>, 8, 3, 0>>());  // 324
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 14>, 16, 3, 0>,
                              MixCfg<MixSched<28, 14>, 8, 2, 0>>());  // 392
  v.push_back(mix_rows_entry<MixCfg<MixSched<24, 20>, 16, 1, 24>,
                              MixCfg<MixSched<24, 20>, 8, 2, 24>>());  // 480
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 20>, 8, 3, 0>,
                              MixCfg<MixSched<28, 20>, 4, 2, 28>>());  // 560
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 24>, 8, 3, 27>,
                              MixCfg<MixSched<27, 24>, 4, 2, 27>>());  // 648
  v.push_back(mix_rows_entry<MixCfg<MixSched<30, 25>, 8, 2, 30>,
                              MixCfg<MixSched<30, 25>, 4, 2, 30>>());  // 750
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 25>, 8, 2, 35>,
                              MixCfg<MixSched<35, 25>, 4, 1, 0>>());  // 875
  v.push_back(mix_rows_entry<MixCfg<MixSched<40, 25>, 4, 3, 0>,
                              MixCfg<MixSched<40, 25>, 2, 3, 0>>());  // 1000
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 9, 9>, 4, 2, 0>,
                              MixCfg<MixSched<14, 9, 9>, 2, 2, 0>>());  // 1134
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 10, 8>, 4, 2, 0>,
                              MixCfg<MixSched<16, 10, 8>, 2, 2, 0>>());  // 1280
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 9, 9>, 4, 2, 0>,
                              MixCfg<MixSched<18, 9, 9>, 2, 2, 0>>());  // 1458
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 12, 9>, 4, 1, 0>,
                              MixCfg<MixSched<15, 12, 9>, 2, 1, 0>>());  // 1620
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 12, 10>, 4, 1, 0>,
                              MixCfg<MixSched<15, 12, 10>, 2, 1, 0>>());  // 1800
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 15, 9>, 2, 2, 0>,
                              MixCfg<MixSched<15, 15, 9>, 2, 1, 0>>());  // 2025
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 14, 9>, 2, 2, 0>,
                              MixCfg<MixSched<18, 14, 9>, 1, 2, 0>>());  // 2268
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 14, 12>, 2, 1, 0>,
                              MixCfg<MixSched<15, 14, 12>, 1, 1, 0>>());  // 2520
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 14, 10>, 2, 2, 0>,
                              MixCfg<MixSched<20, 14, 10>, 1, 2, 0>>());  // 2800
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 21, 7>, 2, 2, 0>,
                              MixCfg<MixSched<21, 21, 7>, 1, 2, 0>>());  // 3087
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 18, 9>, 2, 1, 0>,
                              MixCfg<MixSched<21, 18, 9>, 1, 1, 0>>());  // 3402
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 21, 7>, 2, 1, 0>,
                              MixCfg<MixSched<25, 21, 7>, 1, 1, 0>>());  // 3675
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 16, 14>, 1, 2, 0>,
                              MixCfg<MixSched<18, 16, 14>, 1, 1, 0>>());  // 4032
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 16, 14>, 1, 2, 0>,
                              MixCfg<MixSched<20, 16, 14>, 1, 1, 0>>());  // 4480
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 18, 15>, 1, 2, 0>,
                              MixCfg<MixSched<18, 18, 15>, 1, 1, 0>>());  // 4860
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 15, 14>, 1, 2, 0>,
                              MixCfg<MixSched<25, 15, 14>, 1, 1, 0>>());  // 5250
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 18, 16>, 1, 2, 0>,
                              MixCfg<MixSched<20, 18, 16>, 1, 1, 0>>());  // 5760
  v.push_back(mix_rows_entry64<MixCfg<MixSched<21, 21, 14>, 1, 2, 0>>());  // 6174
  v.push_back(mix_rows_entry64<MixCfg<MixSched<21, 20, 16>, 1, 1, 0>>());  // 6720
  v.push_back(mix_rows_entry64<MixCfg<MixSched<20, 20, 18>, 1, 1, 0>>());  // 7200
  v.push_back(mix_rows_entry64<MixCfg<MixSched<28, 20, 14>, 1, 1, 0>>());  // 7840
  v.push_back(mix_rows_entry64<MixCfg<MixSched<27, 21, 15>, 1, 1, 0>>());  // 8505
  v.push_back(mix_rows_entry64<MixCfg<MixSched<24, 21, 18>, 1, 1, 0>>());  // 9072
  v.push_back(mix_rows_entry64<MixCfg<MixSched<27, 20, 18>, 1, 1, 0>>());  // 9720
  v.push_back(mix_rows_entry64<MixCfg<MixSched<24, 24, 18>, 1, 1, 0>>());  // 10368
  v.push_back(mix_rows_entry64<MixCfg<MixSched<28, 20, 20>, 1, 1, 0>>());  // 11200
  v.push_back(mix_rows_entry64<MixCfg<MixSched<49, 35, 7>, 1, 1, 0>>());  // 12005
}

}  // namespace gfft
