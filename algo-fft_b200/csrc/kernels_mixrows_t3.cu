// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_rows_part_3(std::vector<MixRowsEntry>& v) {
  v.push_back(mix_rows_entry<MixCfg<MixSched<9, 6>, 64, 2, 0>,
                              MixCfg<MixSched<9, 6>, 32, 2, 9>>());  // 54
  v.push_back(mix_rows_entry<MixCfg<MixSched<8, 8>, 64, 2, 0>,
                              MixCfg<MixSched<8, 8>, 32, 3, 0>>());  // 64
  v.push_back(mix_rows_entry<MixCfg<MixSched<10, 8>, 64, 1, 0>,
                              MixCfg<MixSched<10, 8>, 32, 2, 10>>());  // 80
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 8>, 64, 1, 0>,
                              MixCfg<MixSched<12, 8>, 32, 2, 0>>());  // 96
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 9>, 32, 2, 12>,
                              MixCfg<MixSched<12, 9>, 32, 1, 12>>());  // 108
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 9>, 32, 2, 0>,
                              MixCfg<MixSched<14, 9>, 16, 2, 14>>());  // 126
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 12>, 32, 2, 0>,
                              MixCfg<MixSched<12, 12>, 16, 3, 0>>());  // 144
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 9>, 32, 2, 0>,
                              MixCfg<MixSched<18, 9>, 16, 3, 0>>());  // 162
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 9>, 32, 2, 0>,
                              MixCfg<MixSched<21, 9>, 16, 2, 0>>());  // 189
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 14>, 32, 1, 15>,
                              MixCfg<MixSched<15, 14>, 16, 2, 15>>());  // 210
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 15>, 32, 1, 16>,
                              MixCfg<MixSched<16, 15>, 16, 2, 16>>());  // 240
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 14>, 16, 3, 0>,
                              MixCfg<MixSched<18, 14>, 8, 3, 18>>());  // 252
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 16>, 16, 2, 18>,
                              MixCfg<MixSched<18, 16>, 8, 3, 18>>());  // 288
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 16>, 16, 2, 0>,
                              MixCfg<MixSched<20, 16>, 8, 2, 20>>());  // 320
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 14>, 16, 3, 0>,
                              MixCfg<MixSched<25, 14>, 8, 2, 0>>());  // 350
  v.push_back(mix_rows_entry<MixCfg<MixSched<24, 16>, 16, 2, 0>,
                              MixCfg<MixSched<24, 16>, 8, 2, 0>>());  // 384
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 20>, 16, 2, 21>,
                              MixCfg<MixSched<21, 20>, 8, 2, 21>>());  // 420
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 18>, 16, 2, 0>,
                              MixCfg<MixSched<25, 18>, 8, 1, 25>>());  // 450
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 20>, 16, 1, 25>,
                              MixCfg<MixSched<25, 20>, 8, 1, 25>>());  // 500
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 20>, 8, 3, 0>,
                              MixCfg<MixSched<27, 20>, 4, 2, 27>>());  // 540
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 21>, 8, 3, 28>,
                              MixCfg<MixSched<28, 21>, 4, 2, 28>>());  // 588
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 20>, 8, 3, 0>,
                              MixCfg<MixSched<32, 20>, 4, 2, 32>>());  // 640
  v.push_back(mix_rows_entry<MixCfg<MixSched<49, 14>, 8, 3, 0>,
                              MixCfg<MixSched<49, 14>, 4, 3, 0>>());  // 686
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 21>, 8, 2, 0>,
                              MixCfg<MixSched<35, 21>, 4, 2, 0>>());  // 735
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 28>, 8, 3, 0>,
                              MixCfg<MixSched<28, 28>, 4, 2, 0>>());  // 784
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 27>, 8, 2, 32>,
                              MixCfg<MixSched<32, 27>, 4, 2, 32>>());  // 864
  v.push_back(mix_rows_entry<MixCfg<MixSched<30, 30>, 8, 2, 0>,
                              MixCfg<MixSched<30, 30>, 4, 2, 0>>());  // 900
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 28>, 8, 2, 35>,
                              MixCfg<MixSched<35, 28>, 4, 1, 0>>());  // 980
}

}  // namespace gfft
