// Project-written stand-ins for the reference's AffineTransformation and RigidTransformation
// classes (BINDER/src/cpu/{Affine,Rigid}Transformation.h), force-included ahead of the reference
// sources of the test-only library: their .cpp files need Eigen's dynamic matrices and SVD, which
// are not here, and Registration.cpp only constructs them in setAffineTransformation /
// setRigidTransformation, which the checkers never call.  The include guards of the two headers
// are taken, so Registration.cpp compiles unmodified against these.
#pragma once

#include <random>
#include <stdexcept>

#include "Transformation.h"

#define AFFINETRANSFORMATION_H
#define RIGID_TRANSFORMATION_H

class AffineTransformation final : public Transformation {
  public:
    AffineTransformation(const double *, const double *, int, int, int, int, double, double) {
        throw std::runtime_error("the affine transformation is not in the test library");
    }
    double constrain_transformation(const double *, const double *, double *, double *,
                                    int *) override {
        return 0.0;
    }
    void sample_transformation(const double *, const double *, double *, double *, int *,
                               int) override {}
    void set_generator(std::mt19937 &) override {}
};

class RigidTransformation final : public Transformation {
  public:
    RigidTransformation(int, int, int, int, double, double, const double *, const double *,
                        const double *) {
        throw std::runtime_error("the rigid transformation is not in the test library");
    }
    double constrain_transformation(const double *, const double *, double *, double *,
                                    int *) override {
        return 0.0;
    }
    void sample_transformation(const double *, const double *, double *, double *, int *,
                               int) override {}
    void set_generator(std::mt19937 &) override {}
};
