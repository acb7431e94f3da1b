// Scalar bounds of the progressive-sampling stopping rule, evaluated on the
// host from device-reduced values.  Each function restates the reference's
// formula with the same operation order so that the results are the same
// doubles (glibc log/sqrt/pow on both sides).
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

namespace silvan {

// silvan/src/Probabilistic.cpp:80-85
inline double num_samples_bound_fn(double x_, double rho, double delta_, double eps_) {
    double v_x = x_ * (1. - x_);
    double arg_h = eps_ / v_x;
    double denom = v_x * ((1 + arg_h) * log(1 + arg_h) - arg_h);
    return log(2 * rho / (x_ * delta_)) / (denom);
}

// getUpperBoundSamples, silvan/src/Probabilistic.cpp:87-174
inline double upper_bound_samples(double max_bc, double max_var, double avg_spl, double eps,
                                  double delta_bound) {
    double x_hat = 0.;
    double x_hat_low = 0.5 - sqrt(eps / 3.);
    x_hat_low = fmax(x_hat_low, 0.);
    double x_hat_high = 0.5;
    while (x_hat_high - x_hat_low > 0.0001) {
        x_hat = (x_hat_high + x_hat_low) / 2.;
        double v_x = x_hat * (1. - x_hat);
        double arg_h = eps / v_x;
        double f_val = v_x * ((1 + arg_h) * log(1 + arg_h) - arg_h);
        if (f_val <= 2 * pow(eps, 2)) x_hat_high = x_hat;
        else x_hat_low = x_hat;
    }
    x_hat = x_hat_high;
    double x_high = fmin(x_hat, max_bc);
    if (max_var < 0.25) {
        double x_hat_var = 0.5 - sqrt(0.25 - max_var);
        x_high = fmin(x_high, x_hat_var);
    }
    double step = x_high / 1000.;
    double bound_high = num_samples_bound_fn(x_high, avg_spl, delta_bound, eps);
    double bound = bound_high + 1;
    while (bound >= bound_high) {
        double x_low = x_high - step;
        if (x_low > 0.) {
            bound = num_samples_bound_fn(x_low, avg_spl, delta_bound, eps);
            if (bound > bound_high) {
                x_high = x_low;
                bound_high = bound;
            }
        } else {
            bound = bound_high - 1;
        }
    }
    return bound_high;
}

// getUpperBoundTop1BC, silvan/src/Probabilistic.cpp:712-726
inline double upper_bound_top1(double top1_est_bc, double delta, uint64_t num_samples) {
    double log_term = log(1. / delta);
    double c = log_term / (double)num_samples;
    double ub = top1_est_bc + c + sqrt(2 * c * top1_est_bc + pow(c, 2.));
    return fmin(ub, 1.0);
}

// getUpperBoundAvgDiameter, silvan/src/Probabilistic.cpp:729-766
struct AvgDiamBound {
    double avg, ub_b, ub_eb, var, ub;
};
inline AvgDiamBound upper_bound_avg_diameter(const std::vector<uint64_t> &sp_lengths,
                                             int graph_diameter, double delta,
                                             uint64_t num_samples) {
    AvgDiamBound r{};
    double avg = 0.;
    for (int i = 0; i <= graph_diameter; i++)
        avg += (double)i * sp_lengths[i] / (double)(num_samples);
    double log_term = log(1. / delta);
    double c = (graph_diameter - 2) * log_term / (double)num_samples;
    double ub_b = avg + c + sqrt(2 * c * avg + pow(c, 2.));
    double var = 0.;
    for (int i = 0; i <= graph_diameter; i++)
        for (int j = i + 1; j <= graph_diameter; j++)
            var += pow(i - j, 2.0) * sp_lengths[i] / (double)num_samples * sp_lengths[j] /
                   (double)(num_samples - 1);
    log_term = log(2. / delta);
    double ub_eb = avg + 7. / 3. * (graph_diameter - 2) * log_term / (double)num_samples +
                   sqrt(2 * var * log_term / (double)num_samples);
    double ub = fmin(ub_b, ub_eb);
    ub = fmin(ub, (double)(graph_diameter - 2));
    r.avg = avg;
    r.ub_b = ub_b;
    r.ub_eb = ub_eb;
    r.var = var;
    r.ub = ub;
    return r;
}

// get_epsilon_mcrade, silvan/src/Probabilistic.cpp:689-708
inline double epsilon_mcrade(double sup_emp_wimpy_var_, double mcera_, double delta_,
                             double num_samples_, double num_nodes_, int mctrials) {
    mcera_ = fmax(mcera_, 0.);
    double lt = log(5. / delta_) / num_samples_;
    double var_ub = sup_emp_wimpy_var_ + lt + sqrt(pow(lt, 2.) + 2 * lt * sup_emp_wimpy_var_);
    var_ub = fmin(var_ub, 0.25);
    double era_ub = mcera_ + sqrt(4 * sup_emp_wimpy_var_ * lt / (double)mctrials);
    double ra_ub = era_ub + lt + sqrt(pow(lt, 2.) + 2 * lt * era_ub);
    if (num_nodes_ == 1) ra_ub = 0;
    double eps_ub = 2 * ra_ub + sqrt(2 * lt * (var_ub + 4 * ra_ub)) + lt / 3;
    double eps_ub_2 = 2 * ra_ub + sqrt(lt / 2.);
    eps_ub = fmin(eps_ub, eps_ub_2);
    if (num_nodes_ >= 1) {
        double eps_unb = sqrt(2 * var_ub * log(5. / delta_ * num_nodes_) / num_samples_) +
                         log(5. / delta_ * num_nodes_) / num_samples_ / 3;
        eps_ub = fmin(eps_ub, eps_unb);
    }
    return eps_ub;
}

// computeRelBound, silvan/src/Probabilistic.cpp:179-245
inline double relative_bound(double bc_est, double delta, double rho, double m_samples,
                             bool upper, uint32_t n) {
    double upper_ = 1.0, lower_ = 0.;
    if (upper) lower_ = bc_est;
    else upper_ = bc_est;
    for (int i = 0; i < 30; i++) {
        double test_ = (upper_ + lower_) / 2.;
        double v_test_ = test_ * (1. - test_);
        double log_term_ = log(2. / delta * fmin((double)n, rho / test_)) / m_samples;
        double sqrt_term = sqrt(2. * log_term_ * v_test_);
        if (upper) {
            double q = bc_est + log_term_ / 3. + sqrt_term;
            if (q >= test_) lower_ = test_;
            else upper_ = test_;
        } else {
            double q = bc_est - log_term_ / 3. - sqrt_term;
            if (q <= test_) upper_ = test_;
            else lower_ = test_;
        }
    }
    return upper ? upper_ : lower_;
}

}  // namespace silvan
