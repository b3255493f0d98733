// Test infrastructure only.  Stands in for rypath's src/packet_roulette_shared.h when rypath's
// own roulette test program (tests/packet_roulette_tests.cpp) is compiled by oracle/ref.mk, so
// that its known answers run against the oracle's restatement of that header
// (oracle/oracle_math.hpp: EtaScale, account_transmission, rr_prepare) instead of the header
// itself.  The names and meanings are the header's (src/packet_roulette_shared.h:11-108); every
// decision is the oracle's.
#pragma once
#include "oracle_math.hpp"

#include <array>
#include <cstdint>

namespace rypath_packet_roulette {
using Vector = std::array<float, 4>;
inline std::uint32_t bits(float value) { return oracle::fbits(value); }
inline bool finite(float value) { return oracle::rr_finite(value); }
inline bool positive_normal(float value) { return oracle::positive_normal(value); }
inline bool opposite_hemispheres(float a, float b) { return oracle::opposite_hemispheres(a, b); }
struct EtaScale {
    float value = 1;
    bool enabled = true;
};
inline void account_transmission(EtaScale &state, float eta, bool transmission) {
    oracle::EtaScale s{state.value, state.enabled};
    oracle::account_transmission(s, eta, transmission);
    state = {s.value, s.enabled};
}
struct Decision {
    Vector survivor;
    float termination = 0;
    bool eligible = false;
};
inline Decision prepare(Vector beta, const EtaScale &state, unsigned depth) {
    const oracle::Decision d = oracle::rr_prepare(oracle::F4{beta[0], beta[1], beta[2], beta[3]},
                                                  oracle::EtaScale{state.value, state.enabled}, depth);
    return {{d.survivor[0], d.survivor[1], d.survivor[2], d.survivor[3]}, d.termination, d.eligible};
}
// the test program's entry point into the decision: one Bernoulli draw against the prepared
// termination probability, the common survivor factor on survival
inline bool continue_path(Vector &beta, const EtaScale &state, unsigned depth, float u) {
    const Decision decision = prepare(beta, state, depth);
    if (!decision.eligible || !finite(u) || !(u >= 0 && u < 1))
        return true;
    if (u < decision.termination)
        return false;
    beta = decision.survivor;
    return true;
}
} // namespace rypath_packet_roulette
