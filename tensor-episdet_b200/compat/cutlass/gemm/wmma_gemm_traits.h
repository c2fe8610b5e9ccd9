// Interface stand-in, see ../wmma_matrix.h.
#pragma once
#include "../wmma_matrix.h"
