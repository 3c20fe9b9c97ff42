// Entry points whose device paths are not built yet fail loudly.
#include "fold.h"

namespace ef {

FoldOutput chain_fold(Context&, const FoldD&, const std::vector<const Relation*>&, const std::vector<Field>&,
                      const einfold_options&, Budget&) {
  fail(EINFOLD_COMPUTE, "chains are not built yet");
}

}  // namespace ef

