// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_part_3(std::vector<MixEntry>& v) {
  v.push_back(mix_entry<MixCfg<MixSched<9, 6>, 16, 8, 0>,
                         MixCfg<MixSched<9, 6>, 16, 8, 0>,
                         MixCfg<MixSched<9, 6>, 8, 7, 9>,
                         MixCfg<MixSched<9, 6>, 8, 7, 9>>());  // 54
  v.push_back(mix_entry<MixCfg<MixSched<10, 8>, 16, 7, 0>,
                         MixCfg<MixSched<10, 8>, 16, 7, 0>,
                         MixCfg<MixSched<10, 8>, 8, 7, 10>,
                         MixCfg<MixSched<10, 8>, 8, 7, 10>>());  // 80
  v.push_back(mix_entry<MixCfg<MixSched<12, 9>, 16, 5, 12>,
                         MixCfg<MixSched<12, 9>, 16, 5, 12>,
                         MixCfg<MixSched<12, 9>, 8, 6, 12>,
                         MixCfg<MixSched<12, 9>, 8, 6, 12>>());  // 108
  v.push_back(mix_entry<MixCfg<MixSched<12, 12>, 16, 5, 0>,
                         MixCfg<MixSched<12, 12>, 16, 5, 0>,
                         MixCfg<MixSched<12, 12>, 8, 6, 0>,
                         MixCfg<MixSched<12, 12>, 8, 6, 0>>());  // 144
  v.push_back(mix_entry<MixCfg<MixSched<21, 9>, 16, 4, 0>,
                         MixCfg<MixSched<21, 9>, 16, 4, 0>,
                         MixCfg<MixSched<21, 9>, 8, 3, 0>,
                         MixCfg<MixSched<21, 9>, 8, 3, 0>>());  // 189
  v.push_back(mix_entry<MixCfg<MixSched<16, 15>, 16, 3, 16>,
                         MixCfg<MixSched<16, 15>, 16, 3, 16>,
                         MixCfg<MixSched<16, 15>, 8, 4, 16>,
                         MixCfg<MixSched<16, 15>, 8, 4, 16>>());  // 240
  v.push_back(mix_entry<MixCfg<MixSched<18, 16>, 16, 2, 18>,
                         MixCfg<MixSched<18, 16>, 16, 2, 18>,
                         MixCfg<MixSched<18, 16>, 8, 3, 18>,
                         MixCfg<MixSched<18, 16>, 8, 3, 18>>());  // 288
  v.push_back(mix_entry<MixCfg<MixSched<25, 14>, 16, 3, 0>,
                         MixCfg<MixSched<25, 14>, 16, 3, 0>,
                         MixCfg<MixSched<25, 14>, 8, 2, 0>,
                         MixCfg<MixSched<25, 14>, 8, 2, 0>>());  // 350
  v.push_back(mix_entry<MixCfg<MixSched<21, 20>, 16, 2, 21>,
                         MixCfg<MixSched<21, 20>, 16, 2, 21>,
                         MixCfg<MixSched<21, 20>, 8, 2, 21>,
                         MixCfg<MixSched<21, 20>, 8, 2, 21>>());  // 420
  v.push_back(mix_entry<MixCfg<MixSched<25, 20>, 8, 3, 25>,
                         MixCfg<MixSched<25, 20>, 8, 3, 25>,
                         MixCfg<MixSched<25, 20>, 4, 3, 25>,
                         MixCfg<MixSched<25, 20>, 4, 3, 25>>());  // 500
  v.push_back(mix_entry<MixCfg<MixSched<28, 21>, 8, 3, 28>,
                         MixCfg<MixSched<28, 21>, 8, 3, 28>,
                         MixCfg<MixSched<28, 21>, 4, 2, 28>,
                         MixCfg<MixSched<28, 21>, 4, 2, 28>>());  // 588
  v.push_back(mix_entry<MixCfg<MixSched<49, 14>, 8, 3, 0>,
                         MixCfg<MixSched<49, 14>, 8, 3, 0>,
                         MixCfg<MixSched<49, 14>, 4, 3, 0>,
                         MixCfg<MixSched<49, 14>, 4, 3, 0>>());  // 686
  v.push_back(mix_entry<MixCfg<MixSched<28, 28>, 8, 3, 0>,
                         MixCfg<MixSched<28, 28>, 8, 3, 0>,
                         MixCfg<MixSched<28, 28>, 4, 2, 0>,
                         MixCfg<MixSched<28, 28>, 4, 2, 0>>());  // 784
  v.push_back(mix_entry<MixCfg<MixSched<30, 30>, 8, 2, 0>,
                         MixCfg<MixSched<30, 30>, 8, 2, 0>,
                         MixCfg<MixSched<30, 30>, 4, 2, 0>,
                         MixCfg<MixSched<30, 30>, 4, 2, 0>>());  // 900
}

}  // namespace gfft
