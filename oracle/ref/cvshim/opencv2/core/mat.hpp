// TEST INFRASTRUCTURE ONLY: see opencv2/core.hpp of this stand-in.
#pragma once
#include "../core.hpp"
