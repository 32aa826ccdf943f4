/* Stand-in for <mkl.h> (pfft.c:10): only the DFTI part is used on the path. */
#pragma once
#include "mkl_dfti.h"
