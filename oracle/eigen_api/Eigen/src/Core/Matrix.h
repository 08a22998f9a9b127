// See Eigen/Dense in this directory (test infrastructure: a minimal matrix API for the reference harness).
#pragma once
#include "../../Dense"
