// gaffa C++ API on the B200 path: FFA transform shape
// (the reference's include/gaffa/ffa.h:10-13).
#pragma once

#include <cstddef>

namespace gaffa {

struct FfaTransformShape {
  std::size_t rows = 0;
  std::size_t bins = 0;
};

}  // namespace gaffa
