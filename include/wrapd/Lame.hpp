/* Lame.hpp -- wrapd::Lame (the reference's src/Lame.hpp:36-58): Lame
 * parameters from Young's modulus k and Poisson ratio v; preset() uses the
 * reference's 1e7 Pa.  See Math.hpp for this directory's purpose. */
#ifndef WRAPD_COMPAT_LAME_HPP
#define WRAPD_COMPAT_LAME_HPP

namespace wrapd {

class Lame {
public:
    static Lame preset(double poisson) { return Lame(1.0e7, poisson); }
    Lame(double k, double v) : m_mu(k / (2.0 * (1.0 + v))), m_lambda(k * v / ((1.0 + v) * (1.0 - 2.0 * v))) {}
    void mu(double val) { m_mu = val; }
    double mu() const { return m_mu; }
    void lambda(double val) { m_lambda = val; }
    double lambda() const { return m_lambda; }
    /* Young's modulus and Poisson ratio back from (mu, lambda): the solver
     * takes the material as (E, nu). */
    double youngs() const { return m_mu * (3.0 * m_lambda + 2.0 * m_mu) / (m_lambda + m_mu); }
    double poisson() const { return m_lambda / (2.0 * (m_lambda + m_mu)); }

private:
    double m_mu;
    double m_lambda;
};

}  // namespace wrapd

#endif  // WRAPD_COMPAT_LAME_HPP
