/* pre_io_stag.h -- force-included ahead of staggered/io.cpp only: that file
   includes CLI11.hpp before config.h, so the build configuration (which defines
   the `real` macro) must come after CLI11.  TEST INFRASTRUCTURE ONLY. */
#include "CLI11.hpp"
#include "config_stag.h"
