// pmb_learned.cu — sketch features and the strategy-selection MLP.
#include "pmb_groupby.h"
