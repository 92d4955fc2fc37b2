// unary.h of the densecrf_ho API: declared together in densecrf.h.
#pragma once
#include "densecrf.h"
