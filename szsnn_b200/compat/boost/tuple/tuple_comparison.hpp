// The comparisons live with the tuple itself (tuple.hpp).
#pragma once
#include "tuple.hpp"
