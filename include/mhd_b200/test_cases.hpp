// test_cases.hpp -- the reference's test-case API (head/test_cases.hpp:11-72),
// with the configurations this library adds (enum values after OrszagTang).
#pragma once

#include <string>
#include <vector>

#include "types.hpp"

enum class BoundaryType { Periodic, Transmissive, Reflecting, Dirichlet };

struct BoundaryConfig {
    BoundaryType left = BoundaryType::Transmissive;
    BoundaryType right = BoundaryType::Transmissive;
    BoundaryType bottom = BoundaryType::Transmissive;
    BoundaryType top = BoundaryType::Transmissive;
};

enum class CaseId {
    KelvinHelmholtz,  // gamma 1.4, periodic [0,1]x[-1,1]
    ShockBubble,      // Mach 1.22 air / helium, gamma 1.4
    BrioWu,           // Brio-Wu shock tube, gamma 2
    OrszagTang,       // Orszag-Tang on [0,2pi]^2, gamma 5/3
    OrszagTangUnit,   // Orszag-Tang on [0,1]^2 (rho = 25/(36 pi), p = 5/(12 pi)), base 512^2
    ShockBubbleMHD,   // Mach-10 MHD shock - dense bubble on [0,1]^2, gamma 5/3, base 256^2
    BrioWuCFL08       // Brio-Wu 800x4, CFL 0.8, all transmissive
};

struct CaseConfig {
    int nx;
    int ny;
    int ng;
    double x_min;
    double x_max;
    double y_min;
    double y_max;
    double cfl;
    double t_end;
    double gamma;
    BoundaryConfig bc;
    std::vector<double> snapshot_times = {};
    std::vector<std::string> snapshot_tags = {};
};

CaseId parse_case_id(const std::string& case_name);
std::string case_id_to_string(CaseId case_id);
CaseConfig get_case_config(CaseId case_id);
CaseConfig get_case_config(const std::string& case_name);
CaseConfig get_n_case_config(CaseId case_id, int n);
CaseConfig get_n_case_config(const std::string& case_name, int n);
Conserved initial_state_at(CaseId case_id, double x, double y);
Conserved initial_state_at(const std::string& case_name, double x, double y);
