// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_part_1(std::vector<MixEntry>& v) {
  v.push_back(mix_entry<MixCfg<MixSched<7, 7>, 16, 8, 0>,
                         MixCfg<MixSched<7, 7>, 16, 8, 0>,
                         MixCfg<MixSched<7, 7>, 8, 8, 0>,
                         MixCfg<MixSched<7, 7>, 8, 8, 0>>());  // 49
  v.push_back(mix_entry<MixCfg<MixSched<9, 8>, 16, 7, 9>,
                         MixCfg<MixSched<9, 8>, 16, 7, 9>,
                         MixCfg<MixSched<9, 8>, 8, 7, 9>,
                         MixCfg<MixSched<9, 8>, 8, 7, 9>>());  // 72
  v.push_back(mix_entry<MixCfg<MixSched<10, 10>, 16, 6, 0>,
                         MixCfg<MixSched<10, 10>, 16, 6, 0>,
                         MixCfg<MixSched<10, 10>, 8, 7, 0>,
                         MixCfg<MixSched<10, 10>, 8, 7, 0>>());  // 100
  v.push_back(mix_entry<MixCfg<MixSched<15, 9>, 16, 5, 0>,
                         MixCfg<MixSched<15, 9>, 16, 5, 0>,
                         MixCfg<MixSched<15, 9>, 8, 4, 15>,
                         MixCfg<MixSched<15, 9>, 8, 4, 15>>());  // 135
  v.push_back(mix_entry<MixCfg<MixSched<25, 7>, 16, 5, 0>,
                         MixCfg<MixSched<25, 7>, 16, 5, 0>,
                         MixCfg<MixSched<25, 7>, 8, 5, 0>,
                         MixCfg<MixSched<25, 7>, 8, 5, 0>>());  // 175
  v.push_back(mix_entry<MixCfg<MixSched<16, 14>, 16, 3, 16>,
                         MixCfg<MixSched<16, 14>, 16, 3, 16>,
                         MixCfg<MixSched<16, 14>, 8, 4, 16>,
                         MixCfg<MixSched<16, 14>, 8, 4, 16>>());  // 224
  v.push_back(mix_entry<MixCfg<MixSched<18, 15>, 16, 2, 18>,
                         MixCfg<MixSched<18, 15>, 16, 2, 18>,
                         MixCfg<MixSched<18, 15>, 8, 3, 18>,
                         MixCfg<MixSched<18, 15>, 8, 3, 18>>());  // 270
  v.push_back(mix_entry<MixCfg<MixSched<21, 16>, 16, 2, 0>,
                         MixCfg<MixSched<21, 16>, 16, 2, 0>,
                         MixCfg<MixSched<21, 16>, 8, 2, 21>,
                         MixCfg<MixSched<8, 7, 6>, 8, 3, 0>>());  // 336
  v.push_back(mix_entry<MixCfg<MixSched<20, 20>, 16, 2, 0>,
                         MixCfg<MixSched<20, 20>, 16, 2, 0>,
                         MixCfg<MixSched<20, 20>, 8, 2, 0>,
                         MixCfg<MixSched<20, 20>, 8, 2, 0>>());  // 400
  v.push_back(mix_entry<MixCfg<MixSched<27, 18>, 16, 2, 0>,
                         MixCfg<MixSched<27, 18>, 16, 2, 0>,
                         MixCfg<MixSched<27, 18>, 8, 1, 27>,
                         MixCfg<MixSched<27, 18>, 8, 1, 27>>());  // 486
  v.push_back(mix_entry<MixCfg<MixSched<27, 21>, 8, 3, 27>,
                         MixCfg<MixSched<27, 21>, 8, 3, 27>,
                         MixCfg<MixSched<27, 21>, 4, 2, 27>,
                         MixCfg<MixSched<27, 21>, 4, 2, 27>>());  // 567
  v.push_back(mix_entry<MixCfg<MixSched<28, 24>, 8, 3, 28>,
                         MixCfg<MixSched<28, 24>, 8, 3, 28>,
                         MixCfg<MixSched<28, 24>, 4, 2, 28>,
                         MixCfg<MixSched<28, 24>, 4, 2, 28>>());  // 672
  v.push_back(mix_entry<MixCfg<MixSched<28, 27>, 8, 3, 28>,
                         MixCfg<MixSched<28, 27>, 8, 3, 28>,
                         MixCfg<MixSched<28, 27>, 4, 2, 28>,
                         MixCfg<MixSched<28, 27>, 4, 2, 28>>());  // 756
  v.push_back(mix_entry<MixCfg<MixSched<42, 21>, 8, 2, 0>,
                         MixCfg<MixSched<42, 21>, 8, 2, 0>,
                         MixCfg<MixSched<42, 21>, 4, 2, 0>,
                         MixCfg<MixSched<42, 21>, 4, 2, 0>>());  // 882
  v.push_back(mix_entry<MixCfg<MixSched<36, 28>, 8, 2, 36>,
                         MixCfg<MixSched<36, 28>, 8, 2, 36>,
                         MixCfg<MixSched<36, 28>, 4, 1, 0>,
                         MixCfg<MixSched<36, 28>, 4, 1, 0>>());  // 1008
}

}  // namespace gfft
