// ref_host_pin.cpp -- TEST INFRASTRUCTURE: the reference's own hashing and
// probing code, compiled for the host, exported with a C ABI so the tests can
// pin the oracle (and the product's host helpers) to it bit for bit.
//
// Built by oracle/Makefile straight from the reference's headers
// (include/poggers/hash_schemes/murmurhash.cuh, probing_schemes/*.cuh) with
// the host stand-ins in oracle/shim/; the output goes to oracle/_ref/.
#include <cstdint>
#include <poggers/hash_schemes/murmurhash.cuh>
#include <poggers/probing_schemes/double_hashing.cuh>
#include <poggers/probing_schemes/linear_probing.cuh>
#include <poggers/probing_schemes/power_of_two.cuh>
#include <poggers/probing_schemes/xor_power_of_two.cuh>

using poggers::hashers::murmurHasher;

template <class P>
static int run(P &p, uint64_t key, uint64_t tag, uint64_t *out, int cap)
{
    int n = 0;
    for (uint64_t s = p.begin(key); s != p.end() && n < cap; s = p.next(tag)) out[n++] = s;
    return n;
}

extern "C" {

uint64_t refh_murmur64a(uint64_t key, uint64_t seed)
{
    murmurHasher<uint64_t, 1> h;
    h.init(seed);
    return h.hash(key);
}

// kind: 0 double (Max_probes 20), 1 linear (20), 2 power-of-two (2), 3 xor power-of-two (2)
int refh_probe_values(int kind, uint64_t seed, uint64_t key, uint64_t tag, uint64_t *out, int cap)
{
    switch (kind) {
    case 0: { poggers::probing_schemes::doubleHasher<uint64_t, 4, murmurHasher, 20> p(seed); return run(p, key, tag, out, cap); }
    case 1: { poggers::probing_schemes::linearProber<uint64_t, 4, murmurHasher, 20> p(seed); return run(p, key, tag, out, cap); }
    case 2: { poggers::probing_schemes::powerOfTwoHasher<uint64_t, 4, murmurHasher, 2> p(seed); return run(p, key, tag, out, cap); }
    default: { poggers::probing_schemes::XORPowerOfTwoHasher<uint64_t, 4, murmurHasher, 2> p(seed); return run(p, key, tag, out, cap); }
    }
}

}
