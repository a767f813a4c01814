/* pre_io_coll.h -- as pre_io_stag.h, for collocated_AB3/io.cpp.
   TEST INFRASTRUCTURE ONLY. */
#include "CLI11.hpp"
#include "config_coll.h"
