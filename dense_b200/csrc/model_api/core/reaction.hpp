// Include name used by DENSE model headers; the declarations they need are
// in dense_model_api.hpp (one header, so the model files may include these
// names in any order).
#ifndef DENSE_B200_SHIM_CORE_REACTION_HPP
#define DENSE_B200_SHIM_CORE_REACTION_HPP
#include "../dense_model_api.hpp"
#endif
