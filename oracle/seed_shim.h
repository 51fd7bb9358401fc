/*
 * Seed shim for the CPU oracle build of the LGF reference (test
 * infrastructure only).  The reference's default Random() constructor seeds
 * mt19937_64 from std::random_device()+rank (LGF/Math/Random.h:18-22) and its
 * SEED_RNG branch does not compile (LGF/Math/Random.h:13).  Force-included
 * ahead of every reference translation unit, this header pulls in <random>
 * first and then renames random_device, so every default-constructed Random
 * becomes mt19937_64(seed) with seed = $LGF_REF_SEED (default 1) + rank 0.
 * That is the definition of "reference heatbath, seed s" used for the golden
 * inputs.
 */
#ifndef LGF_ORACLE_SEED_SHIM_H
#define LGF_ORACLE_SEED_SHIM_H
#ifdef __cplusplus
#include <random>
#include <cstdlib>
namespace std {
struct lgf_fixed_seed_device {
    typedef unsigned int result_type;
    result_type operator()() const {
        const char* s = std::getenv("LGF_REF_SEED");
        return s ? (result_type)std::strtoul(s, nullptr, 10) : 1u;
    }
};
}  // namespace std
#define random_device lgf_fixed_seed_device
#endif
#endif
