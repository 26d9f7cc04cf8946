// See shared_ptr.hpp: boost::make_shared is std::make_shared here.
#pragma once
#include "shared_ptr.hpp"
