// Stand-in for the CUDA header of this name: see ../esb_ref_shim.h.
#pragma once
#include "../esb_ref_shim.h"
