// Stand-in for the reference's base/reconstruction.h: mvs/utils.h only needs
// Eigen and the basic util headers from it.
#pragma once
#include <Eigen/Core>
#include "util/types.h"
#include "util/math.h"
