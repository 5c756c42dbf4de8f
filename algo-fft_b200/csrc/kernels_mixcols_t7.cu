// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_part_7(std::vector<MixEntry>& v) {
  v.push_back(mix_entry<MixCfg<MixSched<8, 8>, 16, 8, 0>,
                         MixCfg<MixSched<8, 8>, 16, 8, 0>,
                         MixCfg<MixSched<8, 8>, 8, 8, 0>,
                         MixCfg<MixSched<8, 8>, 8, 8, 0>>());  // 64
  v.push_back(mix_entry<MixCfg<MixSched<12, 8>, 16, 7, 0>,
                         MixCfg<MixSched<12, 8>, 16, 7, 0>,
                         MixCfg<MixSched<12, 8>, 8, 8, 0>,
                         MixCfg<MixSched<12, 8>, 8, 8, 0>>());  // 96
  v.push_back(mix_entry<MixCfg<MixSched<14, 9>, 16, 5, 0>,
                         MixCfg<MixSched<14, 9>, 16, 5, 0>,
                         MixCfg<MixSched<14, 9>, 8, 4, 14>,
                         MixCfg<MixSched<14, 9>, 8, 4, 14>>());  // 126
  v.push_back(mix_entry<MixCfg<MixSched<18, 9>, 16, 5, 0>,
                         MixCfg<MixSched<18, 9>, 16, 5, 0>,
                         MixCfg<MixSched<18, 9>, 8, 5, 0>,
                         MixCfg<MixSched<18, 9>, 8, 5, 0>>());  // 162
  v.push_back(mix_entry<MixCfg<MixSched<15, 14>, 16, 3, 15>,
                         MixCfg<MixSched<15, 14>, 16, 3, 15>,
                         MixCfg<MixSched<15, 14>, 8, 4, 15>,
                         MixCfg<MixSched<15, 14>, 8, 4, 15>>());  // 210
  v.push_back(mix_entry<MixCfg<MixSched<18, 14>, 16, 3, 0>,
                         MixCfg<MixSched<18, 14>, 16, 3, 0>,
                         MixCfg<MixSched<18, 14>, 8, 3, 18>,
                         MixCfg<MixSched<18, 14>, 8, 3, 18>>());  // 252
  v.push_back(mix_entry<MixCfg<MixSched<20, 16>, 16, 2, 0>,
                         MixCfg<MixSched<20, 16>, 16, 2, 0>,
                         MixCfg<MixSched<20, 16>, 8, 2, 20>,
                         MixCfg<MixSched<20, 16>, 8, 2, 20>>());  // 320
  v.push_back(mix_entry<MixCfg<MixSched<24, 16>, 16, 2, 0>,
                         MixCfg<MixSched<24, 16>, 16, 2, 0>,
                         MixCfg<MixSched<24, 16>, 8, 2, 0>,
                         MixCfg<MixSched<24, 16>, 8, 2, 0>>());  // 384
  v.push_back(mix_entry<MixCfg<MixSched<25, 18>, 16, 2, 0>,
                         MixCfg<MixSched<25, 18>, 16, 2, 0>,
                         MixCfg<MixSched<25, 18>, 8, 1, 25>,
                         MixCfg<MixSched<25, 18>, 8, 1, 25>>());  // 450
  v.push_back(mix_entry<MixCfg<MixSched<27, 20>, 8, 3, 0>,
                         MixCfg<MixSched<27, 20>, 8, 3, 0>,
                         MixCfg<MixSched<27, 20>, 4, 2, 27>,
                         MixCfg<MixSched<27, 20>, 4, 2, 27>>());  // 540
  v.push_back(mix_entry<MixCfg<MixSched<32, 20>, 8, 3, 0>,
                         MixCfg<MixSched<32, 20>, 8, 3, 0>,
                         MixCfg<MixSched<32, 20>, 4, 2, 32>,
                         MixCfg<MixSched<32, 20>, 4, 2, 32>>());  // 640
  v.push_back(mix_entry<MixCfg<MixSched<35, 21>, 8, 2, 0>,
                         MixCfg<MixSched<35, 21>, 8, 2, 0>,
                         MixCfg<MixSched<35, 21>, 4, 2, 0>,
                         MixCfg<MixSched<35, 21>, 4, 2, 0>>());  // 735
  v.push_back(mix_entry<MixCfg<MixSched<32, 27>, 8, 2, 32>,
                         MixCfg<MixSched<32, 27>, 8, 2, 32>,
                         MixCfg<MixSched<32, 27>, 4, 2, 32>,
                         MixCfg<MixSched<32, 27>, 4, 2, 32>>());  // 864
  v.push_back(mix_entry<MixCfg<MixSched<35, 28>, 8, 2, 35>,
                         MixCfg<MixSched<35, 28>, 8, 2, 35>,
                         MixCfg<MixSched<35, 28>, 4, 1, 0>,
                         MixCfg<MixSched<35, 28>, 4, 1, 0>>());  // 980
}

}  // namespace gfft
