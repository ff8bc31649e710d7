// occupant.cuh — dispatch over a registry of occupants (material models, light kinds).
//
// A registry is an OccupantList of structs, each with a kId (the C ABI value its records
// carry: ptr_material.model, ptr_light.kind).  A family predicate P<M>::value says whether
// M takes part in a dispatch: the build holds it (its census bit) and, for a filtered
// dispatch, it has the trait asked for.  Occupants that do not take part are never
// instantiated, so a per-scene build compiles only the scene's occupants.
#pragma once
#include "common.cuh"

namespace ptx {

template <class... M> struct OccupantList {};

template <template <class> class P, class... M>
__host__ __device__ constexpr bool any_of(OccupantList<M...>) { return (false || ... || P<M>::value); }

// Calls f(M{}) for the occupant M of id `id` among those taking part (P) and returns true;
// false when none matches.  GUARDED: the caller guarantees that `id` belongs to a taking-
// part occupant, so the last one in registry order takes it without a comparison (the final
// else of a generated if-chain; a build holding one candidate calls it directly).  Without
// the guarantee the last candidate is folded only when every occupant the build holds takes
// part (PRESENT names the family's presence predicate).
template <template <class> class P, template <class> class PRESENT, bool GUARDED, class F, class... All>
__device__ __forceinline__ bool dispatch_rest(int, F&, OccupantList<>, OccupantList<All...>) { return false; }
template <template <class> class P, template <class> class PRESENT, bool GUARDED, class F, class M0, class... Ms, class... All>
__device__ __forceinline__ bool dispatch_rest(int id, F& f, OccupantList<M0, Ms...>, OccupantList<All...> all) {
    if constexpr (P<M0>::value) {
        constexpr bool fold = !any_of<P>(OccupantList<Ms...>{}) &&
                              (GUARDED || ((!PRESENT<All>::value || P<All>::value) && ...));
        if constexpr (fold) {
            f(M0{});
            return true;
        } else {
            if (id == M0::kId) {
                f(M0{});
                return true;
            }
        }
    }
    return dispatch_rest<P, PRESENT, GUARDED>(id, f, OccupantList<Ms...>{}, all);
}
template <template <class> class P, template <class> class PRESENT, bool GUARDED, class F, class... M>
__device__ __forceinline__ bool dispatch_occupant(int id, F& f, OccupantList<M...> list) {
    return dispatch_rest<P, PRESENT, GUARDED>(id, f, list, list);
}

// True when `id` belongs to an occupant taking part in P (compared only where needed).
template <template <class> class P>
__device__ __forceinline__ bool occupant_in(int, OccupantList<>) { return false; }
template <template <class> class P, class M0, class... Ms>
__device__ __forceinline__ bool occupant_in(int id, OccupantList<M0, Ms...>) {
    if constexpr (P<M0>::value) {
        if (id == M0::kId) return true;
    }
    return occupant_in<P>(id, OccupantList<Ms...>{});
}

// every id fits a census mask and appears once
template <class... M>
__host__ __device__ constexpr bool ids_distinct(OccupantList<M...>) {
    unsigned bits = 0u;
    bool ok = true;
    ((ok = ok && M::kId >= 0 && M::kId < 32 && !(bits & (1u << M::kId)), bits |= 1u << M::kId), ...);
    return ok;
}

}  // namespace ptx
