// core/fingerprint.h -- the FNV-1a result fingerprints of quarry (src/core/fingerprint.h:16-94):
// one 64-bit word per ray ((hit << 32) | bits(t)) and, per query, (found << 32 | bits(dist2))
// then id + 1; lists fold their length first.  Words are folded whole: h = (h ^ v) * prime.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "core/geometry.h"

struct RayStats {
    uint64_t rays = 0;
    uint64_t hits = 0;
    uint64_t hash = 0xcbf29ce484222325ull;
    double sumT = 0.0;

    void add(const RayHit& h) {
        ++rays;
        uint32_t bits = 0;
        if (h.hit) {
            ++hits;
            sumT += static_cast<double>(h.t);
            std::memcpy(&bits, &h.t, sizeof(bits));
        }
        hash = (hash ^ ((static_cast<uint64_t>(h.hit ? 1u : 0u) << 32) | bits)) * 0x100000001b3ull;
    }

    std::string summary() const {
        char buf[192];
        std::snprintf(buf, sizeof(buf), "rays=%llu hits=%llu sum_t=%.6f hash=0x%016llx",
                      static_cast<unsigned long long>(rays), static_cast<unsigned long long>(hits),
                      sumT, static_cast<unsigned long long>(hash));
        return buf;
    }
};

struct QueryStats {
    uint64_t queries = 0;
    uint64_t results = 0;
    uint64_t hash = 0xcbf29ce484222325ull;
    double sumDist2 = 0.0;

    void add(const ClosestHit& h) {
        ++queries;
        results += h.found ? 1u : 0u;
        mix((static_cast<uint64_t>(h.found ? 1u : 0u) << 32) | bitsOf(h));
        mix(h.found ? static_cast<uint64_t>(h.triangle) + 1u : 0u);
        if (h.found) sumDist2 += static_cast<double>(h.dist2);
    }

    void add(const std::vector<ClosestHit>& list) {
        ++queries;
        results += list.size();
        mix(static_cast<uint64_t>(list.size()));
        for (const ClosestHit& h : list) {
            mix(bitsOf(h));
            mix(static_cast<uint64_t>(h.triangle) + 1u);
            sumDist2 += static_cast<double>(h.dist2);
        }
    }

    std::string summary() const {
        char buf[224];
        std::snprintf(buf, sizeof(buf), "queries=%llu results=%llu sum_dist2=%.6f hash=0x%016llx",
                      static_cast<unsigned long long>(queries),
                      static_cast<unsigned long long>(results), sumDist2,
                      static_cast<unsigned long long>(hash));
        return buf;
    }

private:
    static uint64_t bitsOf(const ClosestHit& h) {
        uint32_t b = 0;
        if (h.found) std::memcpy(&b, &h.dist2, sizeof(b));
        return b;
    }
    void mix(uint64_t v) { hash = (hash ^ v) * 0x100000001b3ull; }
};
