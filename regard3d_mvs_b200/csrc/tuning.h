// Launch-shape table written by the autotuner (regard3d_mvs_b200/autotune.py)
// and read once per process: from $R3DGPU_TUNING_FILE, else from
// tuning_b200.txt in the directory above the library file. Lines:
//   full <nd> <G> <K> <rows>     full-range kernel shape and band rows for exactly nd labels
//   ranged <width> <rows>        band rows of the ranged kernel shape of that label width
//   ranged_wide_frac <f>         share of a tile's pixels allowed wider than its row shape
//   ranged_general_width <w>     ranged tiles whose row shape is at least w labels wide go to the
//                                general kernel
//   path <nd> <G> <K>            chain-pass shape (lanes per chain, label pairs per lane) for exactly
//                                nd labels
// $R3DGPU_TUNING, when set, holds a table's text instead (entries separated by
// newlines or ';', re-read when it changes). Environment overrides
// (R3DGPU_FULL_SHAPE, ...) take precedence; labels without an entry use the
// built-in defaults.
#pragma once

#include <map>

namespace r3dgpu {

struct TunedFull {
  int g, k, rows;
};

struct TunedPath {
  int g, k;
};

struct Tuning {
  std::map<int, TunedFull> full;   // by label count
  std::map<int, TunedPath> path;   // chain-pass shapes by label count
  std::map<int, int> ranged_rows;  // by ranged label width
  double ranged_wide_frac = -1.0;  // < 0: not tuned
  int ranged_general_width = 0;    // 0: not tuned (no ranged tile goes to the general kernel)
  bool loaded = false;
};

const Tuning& tuning();

}  // namespace r3dgpu
