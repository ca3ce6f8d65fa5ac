// Test infrastructure only: schnek/grid.h forwards to grid.hpp.
#include "grid.hpp"
