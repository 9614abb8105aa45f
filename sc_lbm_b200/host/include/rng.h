#ifndef RNG_H
#define RNG_H

#include <random>

/// Uniform random numbers (the reference's include/rng.h:14-31).  The default
/// constructor seeds from std::random_device like the reference; the seeded
/// constructor makes a run reproducible.
class RNG {
public:
    RNG() : gen(std::random_device()()) {}
    explicit RNG(unsigned seed) : gen(seed) {}

    /// Sample of U[dmin, dmax)
    double get_random(const double dmin, const double dmax)
    {
        std::uniform_real_distribution<double> dist(dmin, dmax);
        return dist(gen);
    }

private:
    std::mt19937 gen;
};

#endif
