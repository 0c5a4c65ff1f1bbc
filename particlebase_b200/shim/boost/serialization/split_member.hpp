#pragma once
#include "nvp.hpp"
#define BOOST_SERIALIZATION_SPLIT_MEMBER()
