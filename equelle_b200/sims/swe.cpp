// Explicit shallow-water equations in 2D, written in the form the Equelle
// compiler emits (cf. sintefmath/equelle examples/dsl/swe.equelle, which
// uses the Kurganov-Levy central-upwind flux):
//   - conserved variables q = (w, hu, hv), w = h + b the surface elevation;
//   - a first-order finite-volume Rusanov (local Lax-Friedrichs) flux on the
//     interior faces, along the face normal;
//   - hydrostatic wall fluxes on the boundary faces (reflective walls) and
//     the bathymetry source term from face-midpoint bottom heights, as in
//     the example program;
//   - the example's two-stage Heun step, with dry cells (h <= 0.05) given
//     zero fluxes and wave speeds.
// The time step follows the CFL condition, dt = cfl * min(dx, dy) / max
// over cells of (|u| + sqrt(g h)), from a maxReduce every step; the example
// program reads a list of time steps instead.

#include "equelle/EquelleRuntimeCPU.hpp"

#include <array>

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

    const CollOfScalar h_init = er.inputCollectionOfScalar("h_init", er.allCells());
    const CollOfScalar u_init = er.inputCollectionOfScalar("u_init", er.allCells());
    const CollOfScalar v_init = er.inputCollectionOfScalar("v_init", er.allCells());
    const CollOfScalar b_north = er.inputCollectionOfScalar("b_north", er.allCells());
    const CollOfScalar b_south = er.inputCollectionOfScalar("b_south", er.allCells());
    const CollOfScalar b_east = er.inputCollectionOfScalar("b_east", er.allCells());
    const CollOfScalar b_west = er.inputCollectionOfScalar("b_west", er.allCells());
    const CollOfScalar b_mid = ((((b_north + b_south) + b_east) + b_west) / double(4));
    const Scalar dx = er.inputScalarWithDefault("dx", double(1));
    const Scalar dy = er.inputScalarWithDefault("dy", double(1));
    const Scalar cfl = er.inputScalarWithDefault("cfl", double(0.45));
    const Scalar num_steps = er.inputScalarWithDefault("num_steps", double(200));
    const Scalar gravity = double(9.81);
    const Scalar dry = double(0.05);
    const Scalar dummy = double(1000);
    const CollOfFace int_faces = er.interiorFaces();
    const CollOfFace bound = er.boundaryFaces();
    const CollOfScalar vol = er.norm(er.allCells());
    const CollOfScalar area = er.norm(er.allFaces());
    const CollOfVector int_orientation = er.normal(int_faces);
    const CollOfScalar nx = int_orientation.col(0);
    const CollOfScalar ny = int_orientation.col(1);
    const CollOfCell first = er.firstCell(int_faces);
    const CollOfCell second = er.secondCell(int_faces);
    const CollOfScalar bFirst = er.operatorOn(b_mid, er.allCells(), first);
    const CollOfScalar bSecond = er.operatorOn(b_mid, er.allCells(), second);
    const CollOfVector bound_orientation = er.normal(bound);
    const CollOfCell bound_cells = er.trinaryIf(er.isEmpty(er.firstCell(bound)), er.secondCell(bound), er.firstCell(bound));
    const CollOfScalar bound_b = er.operatorOn(b_mid, er.allCells(), bound_cells);
    const CollOfScalar bound_signX = er.trinaryIf((bound_orientation.col(0) > double(0)), er.operatorExtend(double(1), bound), er.operatorExtend(double(-1), bound));
    const CollOfScalar bound_signY = er.trinaryIf((bound_orientation.col(1) > double(0)), er.operatorExtend(double(1), bound), er.operatorExtend(double(-1), bound));
    const CollOfScalar bx = ((b_east - b_west) / dx);
    const CollOfScalar by = ((b_north - b_south) / dy);

    // flux along the face normal and wave speed, from one side of the faces
    auto sideFlux = [&](const CollOfScalar& w, const CollOfScalar& hu, const CollOfScalar& hv,
                        const CollOfScalar& b) -> std::array<CollOfScalar, 4> {
        const CollOfScalar rawHeight = (w - b);
        const CollOfBool wet = (rawHeight > dry);
        const CollOfScalar height = er.trinaryIf(wet, rawHeight, er.operatorExtend(dummy, int_faces));
        const CollOfScalar qn = ((hu * nx) + (hv * ny));
        const CollOfScalar un = (qn / height);
        const CollOfScalar pressure = ((double(0.5) * gravity) * (height * height));
        const CollOfScalar zero = er.operatorExtend(double(0), int_faces);
        const CollOfScalar f0 = er.trinaryIf(wet, qn, zero);
        const CollOfScalar f1 = er.trinaryIf(wet, ((hu * un) + (pressure * nx)), zero);
        const CollOfScalar f2 = er.trinaryIf(wet, ((hv * un) + (pressure * ny)), zero);
        const CollOfScalar speed = er.trinaryIf(wet, (er.sqrt((un * un)) + er.sqrt((gravity * height))), zero);
        return {f0, f1, f2, speed};
    };

    // Rusanov fluxes on the interior faces, wall fluxes on the boundary,
    // times the face areas, on all faces
    auto getFlux = [&](const CollOfScalar& w, const CollOfScalar& hu, const CollOfScalar& hv) -> std::array<CollOfScalar, 3> {
        const CollOfScalar wL = er.operatorOn(w, er.allCells(), first);
        const CollOfScalar huL = er.operatorOn(hu, er.allCells(), first);
        const CollOfScalar hvL = er.operatorOn(hv, er.allCells(), first);
        const CollOfScalar wR = er.operatorOn(w, er.allCells(), second);
        const CollOfScalar huR = er.operatorOn(hu, er.allCells(), second);
        const CollOfScalar hvR = er.operatorOn(hv, er.allCells(), second);
        const std::array<CollOfScalar, 4> fL = sideFlux(wL, huL, hvL, bFirst);
        const std::array<CollOfScalar, 4> fR = sideFlux(wR, huR, hvR, bSecond);
        const CollOfScalar a = er.trinaryIf((fL[3] > fR[3]), fL[3], fR[3]);
        const CollOfScalar intFlux0 = ((double(0.5) * (fL[0] + fR[0])) - ((double(0.5) * a) * (wR - wL)));
        const CollOfScalar intFlux1 = ((double(0.5) * (fL[1] + fR[1])) - ((double(0.5) * a) * (huR - huL)));
        const CollOfScalar intFlux2 = ((double(0.5) * (fL[2] + fR[2])) - ((double(0.5) * a) * (hvR - hvL)));
        const CollOfScalar bound_height = (er.operatorOn(w, er.allCells(), bound_cells) - bound_b);
        const CollOfScalar b_flux = er.trinaryIf((bound_height > dry), ((double(0.5) * gravity) * (bound_height * bound_height)), er.operatorExtend(double(0), bound));
        const CollOfScalar boundFlux1 = ((er.sqrt((bound_orientation.col(0) * bound_orientation.col(0))) * b_flux) * bound_signX);
        const CollOfScalar boundFlux2 = ((er.sqrt((bound_orientation.col(1) * bound_orientation.col(1))) * b_flux) * bound_signY);
        const CollOfScalar all0 = (er.operatorExtend(intFlux0, int_faces, er.allFaces()) * area);
        const CollOfScalar all1 = ((er.operatorExtend(intFlux1, int_faces, er.allFaces()) + er.operatorExtend(boundFlux1, bound, er.allFaces())) * area);
        const CollOfScalar all2 = ((er.operatorExtend(intFlux2, int_faces, er.allFaces()) + er.operatorExtend(boundFlux2, bound, er.allFaces())) * area);
        return {all0, all1, all2};
    };

    // bathymetry source terms of the momentum equations
    auto sourceTerm = [&](const CollOfScalar& w) -> std::array<CollOfScalar, 2> {
        const CollOfScalar secondTerm_x = (((w - b_east) + (w - b_west)) / double(2));
        const CollOfScalar secondTerm_y = (((w - b_north) + (w - b_south)) / double(2));
        const CollOfScalar dryTerm = er.trinaryIf(((w - b_mid) > dry), er.operatorExtend(double(1), er.allCells()), er.operatorExtend(double(0), er.allCells()));
        return {((((-gravity) * bx) * secondTerm_x) * dryTerm), ((((-gravity) * by) * secondTerm_y) * dryTerm)};
    };

    // forward Euler stage q + dt/vol (-div F(q) + vol S(q))
    auto eulerStage = [&](const CollOfScalar& w, const CollOfScalar& hu, const CollOfScalar& hv, const Scalar& dt) -> std::array<CollOfScalar, 3> {
        const std::array<CollOfScalar, 3> flux = getFlux(w, hu, hv);
        const std::array<CollOfScalar, 2> source = sourceTerm(w);
        const CollOfScalar w1 = (w + ((dt / vol) * (-er.divergence(flux[0]))));
        const CollOfScalar hu1 = (hu + ((dt / vol) * ((-er.divergence(flux[1])) + (vol * source[0]))));
        const CollOfScalar hv1 = (hv + ((dt / vol) * ((-er.divergence(flux[2])) + (vol * source[1]))));
        return {w1, hu1, hv1};
    };

    // largest wave speed over the cells (dry cells: 0)
    auto maxSpeed = [&](const CollOfScalar& w, const CollOfScalar& hu, const CollOfScalar& hv) -> Scalar {
        const CollOfScalar rawHeight = (w - b_mid);
        const CollOfBool wet = (rawHeight > dry);
        const CollOfScalar height = er.trinaryIf(wet, rawHeight, er.operatorExtend(dummy, er.allCells()));
        const CollOfScalar u = (hu / height);
        const CollOfScalar v = (hv / height);
        const CollOfScalar speed = er.trinaryIf(wet, (er.sqrt(((u * u) + (v * v))) + er.sqrt((gravity * height))), er.operatorExtend(double(0), er.allCells()));
        return er.maxReduce(speed);
    };

    CollOfScalar w0 = (h_init + b_mid);
    CollOfScalar hu0 = (h_init * u_init);
    CollOfScalar hv0 = (h_init * v_init);
    er.output("q1", w0);
    er.output("q2", hu0);
    er.output("q3", hv0);
    const Scalar h_min = (dx < dy) ? dx : dy;
    for (int step = 0; step < int(num_steps); ++step) {
        const Scalar dt = ((cfl * h_min) / maxSpeed(w0, hu0, hv0));
        const std::array<CollOfScalar, 3> qs = eulerStage(w0, hu0, hv0, dt);
        const std::array<CollOfScalar, 3> qss = eulerStage(qs[0], qs[1], qs[2], dt);
        const CollOfScalar w = ((double(0.5) * w0) + (double(0.5) * qss[0]));
        const CollOfScalar hu = ((double(0.5) * hu0) + (double(0.5) * qss[1]));
        const CollOfScalar hv = ((double(0.5) * hv0) + (double(0.5) * qss[2]));
        er.output("q1", w);
        er.output("q2", hu);
        er.output("q3", hv);
        w0 = w;
        hu0 = hu;
        hv0 = hv;
    }

    // ============= Generated code ends here ================
}

void ensureRequirements(const equelle::EquelleRuntimeCPU& er)
{
    er.ensureGridDimensionMin(2);
}
