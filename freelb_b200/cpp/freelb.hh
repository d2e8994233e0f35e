// freelb.hh -- companion of freelb.h.  The reference splits declarations
// (freelb.h) and definitions (freelb.hh); every definition of the B200 host
// classes is in freelb.h, so programs that include both compile unchanged.
#pragma once
#include "freelb.h"
