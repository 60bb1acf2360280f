// Pass-kernel instantiations: length family p2, double, 2 field(s) per pass.
#include "gpe_sizes.h"
#define GPE_R double
#define GPE_SFX d
#define GPE_FAM p2
#define GPE_NF 2
#define GPE_SIZES(X) GPE_SIZES_p2(X)
#define GPE_TUNED(X) GPE_TUNED_p2(X)
#include "gpe_inst_body.cuh"
