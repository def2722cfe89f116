// devicearray.h -- name kept from the reference's include/ tree so that code written against
// eljens/multigrid-poisson compiles unchanged; everything lives in poisson_facade.h.
#pragma once
#include "poisson_facade.h"
