
// Implicit heat equation in the form the Equelle compiler emits for a
// conduction program with Dirichlet faces (cf. sintefmath/equelle
// examples/app/out_heateq.cpp): two-point conductivities on interior and
// Dirichlet boundary faces, zero flux on the other boundary faces, one
// newtonSolve per time step.

#include "equelle/EquelleRuntimeCPU.hpp"

void equelleGeneratedCode(equelle::EquelleRuntimeCPU& er);
void ensureRequirements(const equelle::EquelleRuntimeCPU& er);

#ifndef EQUELLE_NO_MAIN
int main(int argc, char** argv)
{
    Opm::ParameterGroup param(argc, argv, false);
    equelle::EquelleRuntimeCPU er(param);
    equelleGeneratedCode(er);
    return 0;
}
#endif  // EQUELLE_NO_MAIN

void equelleGeneratedCode(equelle::EquelleRuntimeCPU& er)
{
    using namespace equelle;
    ensureRequirements(er);

    // ============= Generated code starts here ================

    const Scalar k = er.inputScalarWithDefault("k", double(0.3));
    const Scalar cv = er.inputScalarWithDefault("cv", double(1));
    const CollOfFace inner_faces = er.interiorFaces();
    const CollOfScalar inner_cond =
        (k * (er.norm(inner_faces) / er.norm((er.centroid(er.firstCell(inner_faces)) - er.centroid(er.secondCell(inner_faces))))));
    auto innerFlux = [&](const CollOfScalar& u) -> CollOfScalar { return (-inner_cond * er.gradient(u)); };
    const CollOfFace dirichlet_faces = er.inputDomainSubsetOf("dir_boundary", er.boundaryFaces());
    const CollOfScalar dirichlet_value = er.inputCollectionOfScalar("dir_val", dirichlet_faces);
    const CollOfFace outer_faces = er.boundaryFaces();
    const CollOfBool outside_first = er.isEmpty(er.firstCell(outer_faces));
    const CollOfCell outer_cells = er.trinaryIf(outside_first, er.secondCell(outer_faces), er.firstCell(outer_faces));
    const CollOfScalar outer_sign =
        er.trinaryIf(outside_first, er.operatorExtend(-double(1), outer_faces), er.operatorExtend(double(1), outer_faces));
    const CollOfScalar outer_cond =
        (k * (er.norm(outer_faces) / er.norm((er.centroid(outer_faces) - er.centroid(outer_cells)))));
    const CollOfCell dirichlet_cells = er.operatorOn(outer_cells, er.boundaryFaces(), dirichlet_faces);
    const CollOfScalar dirichlet_coef =
        (er.operatorOn(outer_cond, er.boundaryFaces(), dirichlet_faces) * er.operatorOn(outer_sign, er.boundaryFaces(), dirichlet_faces));
    auto dirichletFlux = [&](const CollOfScalar& u) -> CollOfScalar {
        const CollOfScalar u_inside = er.operatorOn(u, er.allCells(), dirichlet_cells);
        const CollOfScalar flux = (dirichlet_coef * (u_inside - dirichlet_value));
        return er.operatorExtend(flux, dirichlet_faces, er.boundaryFaces());
    };
    const CollOfScalar volume = er.norm(er.allCells());
    auto heatResidual = [&](const CollOfScalar& u, const CollOfScalar& u_old, const Scalar& dt) -> CollOfScalar {
        const CollOfScalar all_fluxes = (er.operatorExtend(innerFlux(u), er.interiorFaces(), er.allFaces()) +
                                         er.operatorExtend(dirichletFlux(u), er.boundaryFaces(), er.allFaces()));
        return ((u - u_old) + ((dt / (cv * volume)) * er.divergence(all_fluxes)));
    };
    const CollOfScalar u_initial = er.inputCollectionOfScalar("u_initial", er.allCells());
    const SeqOfScalar timesteps = er.inputSequenceOfScalar("timesteps");
    auto u_old = u_initial;
    er.output("u", u_old);
    for (const Scalar& dt : timesteps) {
        auto residualAtStep = [&](const CollOfScalar& u) -> CollOfScalar { return heatResidual(u, u_old, dt); };
        const CollOfScalar u = er.newtonSolve(residualAtStep, u_old);
        er.output("u", u);
        er.output("maximum of u", er.maxReduce(u));
        u_old = u;
    }

    // ============= Generated code ends here ================
}

void ensureRequirements(const equelle::EquelleRuntimeCPU& er)
{
    (void)er;
}
