// ceos_oracle_visco.cpp -- TEST INFRASTRUCTURE ONLY.
// Restatement of the reference's variational viscoelastic matrix model
// (ConstitutiveModelsLibrary/ModViscoelasticMatrix.f90).  Filled in below.
int visco_var_update(const double* p, const double* F, double dt, const double* st_old,
                     double* st_new, double* sig, double* D) {
    (void)p; (void)F; (void)dt; (void)st_old; (void)st_new; (void)sig; (void)D;
    return 9;
}
