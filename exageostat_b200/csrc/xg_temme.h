/* The order-only constants of Temme's series for K_nu (kbessel.cuh): mu =
 * nu - n, n = round(nu), |mu| <= 1/2; gamma1 / gamma2 of Temme's paper (from
 * the Taylor polynomials of 1/Gamma), Gamma(1 + mu), Gamma(1 - mu),
 * pi mu / sin(pi mu) and 2^mu.  Plain data, so the covariance generators can
 * carry them in their kernel parameters (xg_temme_consts fills them). */
#ifndef EXAGEOSTAT_B200_XG_TEMME_H
#define EXAGEOSTAT_B200_XG_TEMME_H

struct XgTemme {
    double mu, m2, gamma1, gamma2, grp, grm, pimu_sin, two_mu;
    int n;
};

#endif
