// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_rows_part_3(std::vector<MixRowsEntry>& v) {
  v.push_back(mix_rows_entry<MixCfg<MixSched<9, 6>, 64, 2, 0>,
                              MixCfg<MixSched<9, 6>, 32, 2, 9>>());  // 54
  v.push_back(mix_rows_entry<MixCfg<MixSched<10, 8>, 64, 1, 0>,
                              MixCfg<MixSched<10, 8>, 32, 2, 10>>());  // 80
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 9>, 32, 2, 12>,
                              MixCfg<MixSched<12, 9>, 32, 1, 12>>());  // 108
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 12>, 32, 2, 0>,
                              MixCfg<MixSched<12, 12>, 16, 3, 0>>());  // 144
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 9>, 32, 2, 0>,
                              MixCfg<MixSched<21, 9>, 16, 2, 0>>());  // 189
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 15>, 32, 1, 16>,
                              MixCfg<MixSched<16, 15>, 16, 2, 16>>());  // 240
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 16>, 16, 2, 18>,
                              MixCfg<MixSched<18, 16>, 8, 3, 18>>());  // 288
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 14>, 16, 3, 0>,
                              MixCfg<MixSched<25, 14>, 8, 2, 0>>());  // 350
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 20>, 16, 2, 21>,
                              MixCfg<MixSched<21, 20>, 8, 2, 21>>());  // 420
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 20>, 16, 1, 25>,
                              MixCfg<MixSched<25, 20>, 8, 1, 25>>());  // 500
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 21>, 8, 3, 28>,
                              MixCfg<MixSched<28, 21>, 4, 2, 28>>());  // 588
  v.push_back(mix_rows_entry<MixCfg<MixSched<49, 14>, 8, 3, 0>,
                              MixCfg<MixSched<49, 14>, 4, 3, 0>>());  // 686
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 28>, 8, 3, 0>,
                              MixCfg<MixSched<28, 28>, 4, 2, 0>>());  // 784
  v.push_back(mix_rows_entry<MixCfg<MixSched<30, 30>, 8, 2, 0>,
                              MixCfg<MixSched<30, 30>, 4, 2, 0>>());  // 900
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 7, 7>, 4, 3, 0>,
                              MixCfg<MixSched<21, 7, 7>, 2, 3, 0>>());  // 1029
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 10, 10>, 4, 1, 0>,
                              MixCfg<MixSched<12, 10, 10>, 2, 2, 0>>());  // 1200
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 12, 8>, 4, 1, 0>,
                              MixCfg<MixSched<14, 12, 8>, 2, 2, 0>>());  // 1344
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 12, 9>, 4, 1, 0>,
                              MixCfg<MixSched<14, 12, 9>, 2, 1, 0>>());  // 1512
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 7, 7>, 4, 2, 0>,
                              MixCfg<MixSched<35, 7, 7>, 2, 2, 0>>());  // 1715
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 12, 10>, 4, 1, 0>,
                              MixCfg<MixSched<16, 12, 10>, 2, 1, 0>>());  // 1920
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 12, 12>, 2, 2, 0>,
                              MixCfg<MixSched<15, 12, 12>, 1, 2, 0>>());  // 2160
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 15, 10>, 2, 2, 0>,
                              MixCfg<MixSched<16, 15, 10>, 1, 2, 0>>());  // 2400
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 15, 7>, 2, 2, 0>,
                              MixCfg<MixSched<25, 15, 7>, 1, 2, 0>>());  // 2625
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 18, 9>, 2, 2, 0>,
                              MixCfg<MixSched<18, 18, 9>, 1, 2, 0>>());  // 2916
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 15, 14>, 2, 1, 0>,
                              MixCfg<MixSched<15, 15, 14>, 1, 1, 0>>());  // 3150
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 14, 10>, 2, 2, 0>,
                              MixCfg<MixSched<25, 14, 10>, 1, 2, 0>>());  // 3500
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 16, 15>, 2, 1, 0>,
                              MixCfg<MixSched<16, 16, 15>, 1, 1, 0>>());  // 3840
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 15, 14>, 1, 2, 0>,
                              MixCfg<MixSched<20, 15, 14>, 1, 1, 0>>());  // 4200
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 16, 16>, 1, 2, 0>,
                              MixCfg<MixSched<18, 16, 16>, 1, 1, 0>>());  // 4608
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 18, 14>, 1, 2, 0>,
                              MixCfg<MixSched<20, 18, 14>, 1, 1, 0>>());  // 5040
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 18, 15>, 1, 2, 0>,
                              MixCfg<MixSched<20, 18, 15>, 1, 1, 0>>());  // 5400
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 20, 15>, 1, 2, 0>,
                              MixCfg<MixSched<20, 20, 15>, 1, 1, 0>>());  // 6000
  v.push_back(mix_rows_entry64<MixCfg<MixSched<21, 20, 15>, 1, 1, 0>>());  // 6300
  v.push_back(mix_rows_entry64<MixCfg<MixSched<35, 14, 14>, 1, 2, 0>>());  // 6860
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 21, 14>, 1, 1, 0>>());  // 7350
  v.push_back(mix_rows_entry64<MixCfg<MixSched<20, 20, 20>, 1, 1, 0>>());  // 8000
  v.push_back(mix_rows_entry64<MixCfg<MixSched<27, 18, 18>, 1, 1, 0>>());  // 8748
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 25, 15>, 1, 1, 0>>());  // 9375
  v.push_back(mix_rows_entry64<MixCfg<MixSched<24, 21, 20>, 1, 1, 0>>());  // 10080
  v.push_back(mix_rows_entry64<MixCfg<MixSched<28, 24, 16>, 1, 1, 0>>());  // 10752
  v.push_back(mix_rows_entry64<MixCfg<MixSched<24, 24, 20>, 1, 1, 0>>());  // 11520
  v.push_back(mix_rows_entry64<MixCfg<MixSched<35, 25, 14>, 1, 1, 0>>());  // 12250
}

}  // namespace gfft
