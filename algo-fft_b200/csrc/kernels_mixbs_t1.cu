// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_bs_part_1(std::vector<MixBsEntry>& v) {
  v.push_back(mix_bs_entry<MixCfg<MixSched<14, 8>, 16, 7, 0>,
                            MixCfg<MixSched<14, 8>, 8, 8, 0>>());  // 112
  v.push_back(mix_bs_entry<MixCfg<MixSched<16, 10>, 16, 5, 0>,
                            MixCfg<MixSched<16, 10>, 8, 4, 16>>());  // 160
  v.push_back(mix_bs_entry<MixCfg<MixSched<16, 15>, 16, 3, 16>,
                            MixCfg<MixSched<16, 15>, 8, 4, 16>>());  // 240
  v.push_back(mix_bs_entry<MixCfg<MixSched<20, 16>, 16, 2, 0>,
                            MixCfg<MixSched<20, 16>, 8, 2, 20>>());  // 320
  v.push_back(mix_bs_entry<MixCfg<MixSched<20, 20>, 16, 2, 0>,
                            MixCfg<MixSched<20, 20>, 8, 2, 0>>());  // 400
  v.push_back(mix_bs_entry<MixCfg<MixSched<10, 8, 6>, 8, 3, 0>,
                            MixCfg<MixSched<24, 20>, 8, 2, 24>>());  // 480
}

}  // namespace gfft
