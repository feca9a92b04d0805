// pmb_sort.cu — packed-key LSD radix sort + segmented reduce (group-by sort strategy).
#include "pmb_groupby.h"
