// Pass-kernel instantiations: length family p9b, float, 2 field(s) per pass.
#include "gpe_sizes.h"
#define GPE_R float
#define GPE_PAIRED 1
#define GPE_SFX f
#define GPE_FAM p9b
#define GPE_NF 2
#define GPE_SIZES(X) GPE_SIZES_p9b(X)
#define GPE_TUNED(X) GPE_TUNED_p9b(X)
#include "gpe_inst_body.cuh"
