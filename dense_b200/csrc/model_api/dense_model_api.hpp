// Model API of the DENSE deterministic engine, compiled from a DENSE model
// directory (specie_list.hpp, reactions_list.hpp, reaction_deltas.hpp,
// model_impl.hpp) without changing those files.
//
// DENSE's model headers include "core/reaction.hpp", "core/specie.hpp",
// "core/model.hpp", "sim/base.hpp" and "utility/common_utils.hpp"; this tree
// ships its own headers under those names, and each of them includes this
// file.  What the model files need from them is restated here:
//
//   * enum Species / specie_id / NUM_SPECIES and Critical_Species_ID
//     (rcrit_<name>) built from specie_list.hpp, in list order
//     (DENSE core/specie.hpp:10-37);
//   * enum Reaction_ID / reaction_id / NUM_REACTIONS and delay_reaction_id
//     (dreact_<name>) built from reactions_list.hpp (core/reaction.hpp:12-36);
//   * NUM_PARAMS and the parameter layout [rates | delays | critical values]
//     (core/parameter_set.hpp:9-13);
//   * template reaction<RID> with the member template
//     active_rate<Ctxt>(Ctxt const&) that model_impl.hpp specialises
//     (core/reaction.hpp:58-65).  Here it is __host__ __device__, so the same
//     specialisations compile for the CPU set-up code and for the sm_100a step
//     kernel;
//   * STATIC_VAR, used by reaction_deltas.hpp for the stoichiometry tables.
//     It expands to `static constexpr` (plus __device__ under nvcc), so the
//     step kernel sees every delta as a compile-time constant and keeps the
//     per-species delta accumulators in registers.
//
// The arithmetic type is `Real`, double unless DENSE_B200_REAL names another
// floating type (the FP32 engine translation unit compiles the model with
// float, DENSE's own `Real` being configurable the same way,
// utility/configurable.hpp:30-45).
#ifndef DENSE_B200_MODEL_API_HPP
#define DENSE_B200_MODEL_API_HPP

#include <cstddef>
#include <cmath>

#ifdef __CUDACC__
#define DENSE_HD __host__ __device__
#define DENSE_DEVICE_VAR __device__
#else
#define DENSE_HD
#define DENSE_DEVICE_VAR
#endif

// Execution-space macros that DENSE model code may use
// (DENSE utility/cuda.hpp:8-54 defines the same names).
#ifndef CUDA_AGNOSTIC
#define CUDA_AGNOSTIC DENSE_HD
#endif
#ifndef CUDA_HOST
#ifdef __CUDACC__
#define CUDA_HOST __host__
#define CUDA_DEVICE __device__
#else
#define CUDA_HOST
#define CUDA_DEVICE
#endif
#endif

#ifndef STATIC_VAR
#define STATIC_VAR static constexpr DENSE_DEVICE_VAR
#endif

#ifndef DENSE_B200_REAL
#define DENSE_B200_REAL double
#endif

namespace dense {
using Real = DENSE_B200_REAL;
using Natural = int;
using Index = std::ptrdiff_t;
}  // namespace dense
using dense::Natural;
using dense::Real;
using RATETYPE = ::Real;

// ---------------------------------------------------------------- species
enum Species {
#define SPECIE(name) name,
#define CRITICAL_SPECIE(name) name,
#include "specie_list.hpp"
#undef CRITICAL_SPECIE
#undef SPECIE
  size
};
constexpr int NUM_SPECIES = Species::size;
using specie_id = Species;

enum Critical_Species_ID {
#define SPECIE(name)
#define CRITICAL_SPECIE(name) rcrit_##name,
#include "specie_list.hpp"
#undef SPECIE
#undef CRITICAL_SPECIE
  NUM_CRITICAL_SPECIES
};
using critspecie_id = Critical_Species_ID;

// Which species are critical, in species order (host-side set-up only).
constexpr int dense_critical_species_of[NUM_CRITICAL_SPECIES + 1] = {
#define SPECIE(name)
#define CRITICAL_SPECIE(name) name,
#include "specie_list.hpp"
#undef SPECIE
#undef CRITICAL_SPECIE
    -1};

// -------------------------------------------------------------- reactions
enum Reaction_ID {
#define REACTION(name) name,
#include "reactions_list.hpp"
#undef REACTION
  Reaction_ID_size
};
constexpr int NUM_REACTIONS = Reaction_ID_size;
using reaction_id = Reaction_ID;

enum delay_reaction_id {
#define REACTION(name)
#define DELAY_REACTION(name) dreact_##name,
#include "reactions_list.hpp"
#undef REACTION
#undef DELAY_REACTION
  NUM_DELAY_REACTIONS
};

// reaction id of each delay reaction, in delay-reaction order.
constexpr int dense_delay_reaction_of[NUM_DELAY_REACTIONS + 1] = {
#define REACTION(name)
#define DELAY_REACTION(name) name,
#include "reactions_list.hpp"
#undef REACTION
#undef DELAY_REACTION
    -1};

// ------------------------------------------------------------- parameters
constexpr int NUM_PARAMS = NUM_CRITICAL_SPECIES + NUM_REACTIONS + NUM_DELAY_REACTIONS;
constexpr int rate_constants_offset_ = 0;
constexpr int delays_offset_ = rate_constants_offset_ + NUM_REACTIONS;
constexpr int critical_values_offset_ = delays_offset_ + NUM_DELAY_REACTIONS;

// --------------------------------------------------------- reaction rates
// model_impl.hpp provides one explicit specialisation of active_rate per
// reaction.  The primary template is declared only.
template <reaction_id RID>
class reaction {
 public:
  template <class Ctxt>
  DENSE_HD static Real active_rate(Ctxt const& c);
};

// Names, for CSV headers and reports.
static const char* const dense_specie_names[NUM_SPECIES + 1] = {
#define SPECIE(name) #name,
#define CRITICAL_SPECIE(name) #name,
#include "specie_list.hpp"
#undef CRITICAL_SPECIE
#undef SPECIE
    nullptr};

static const char* const dense_reaction_names[NUM_REACTIONS + 1] = {
#define REACTION(name) #name,
#include "reactions_list.hpp"
#undef REACTION
    nullptr};

#endif  // DENSE_B200_MODEL_API_HPP
