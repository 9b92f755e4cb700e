"""Generated-style simulator programs over the Python runtime mirror.

Each function is written the way the Equelle compiler emits C++ for the
corresponding .equelle program (a flat sequence of runtime calls with
lambdas for Equelle functions), so the same op stream runs on the device
library and on the CPU oracle.  The C++ twins in equelle_b200/sims/ are
what bench.py runs.

  heat_equation      implicit heat equation with Dirichlet faces
                     (the program sintefmath/equelle examples/app/
                     out_heateq.cpp was generated from)
  two_phase          fully implicit incompressible oil-water flow with
                     phase upwinding (examples/app/
                     out_twophase_fully_implicit.cpp), Corey exponent
                     as a parameter
"""
import numpy as np

from . import capi


def heat_equation(er, k, cv, u_initial, dir_faces, dir_val, timesteps, on_step=None):
    """Returns the list of u fields after each step (host arrays)."""
    ifaces = er.interiorFaces()
    first = er.firstCell(ifaces)
    second = er.secondCell(ifaces)
    itrans = k * (er.norm(ifaces) / er.norm(er.centroid(first) - er.centroid(second)))

    def interior_flux(u):
        return -itrans * er.gradient(u)

    dir_boundary = er.entity_set(capi.FACES, dir_faces)
    dir_value = er.collection(dir_val)
    bf = er.boundaryFaces()
    bf_cells = er.trinaryIf(er.isEmpty(er.firstCell(bf)), er.secondCell(bf), er.firstCell(bf))
    bf_sign = er.trinaryIf(er.isEmpty(er.firstCell(bf)), er.operatorExtend(-1.0, bf), er.operatorExtend(1.0, bf))
    btrans = k * (er.norm(bf) / er.norm(er.centroid(bf) - er.centroid(bf_cells)))
    dir_cells = er.operatorOn(bf_cells, er.boundaryFaces(), dir_boundary)
    dir_sign = er.operatorOn(bf_sign, er.boundaryFaces(), dir_boundary)
    dir_trans = er.operatorOn(btrans, er.boundaryFaces(), dir_boundary)

    def boundary_flux(u):
        u_dirbdycells = er.operatorOn(u, er.allCells(), dir_cells)
        dir_fluxes = (dir_trans * dir_sign) * (u_dirbdycells - dir_value)
        return er.operatorExtend(dir_fluxes, dir_boundary, er.boundaryFaces())

    vol = er.norm(er.allCells())

    def residual(u, u0, dt):
        ifluxes = interior_flux(u)
        bfluxes = boundary_flux(u)
        fluxes = (er.operatorExtend(ifluxes, er.interiorFaces(), er.allFaces())
                  + er.operatorExtend(bfluxes, er.boundaryFaces(), er.allFaces()))
        return (u - u0) + ((dt / (cv * vol)) * er.divergence(fluxes))

    u0 = er.collection(u_initial)
    out = []
    for dt in timesteps:
        u = er.newtonSolve(lambda uu: residual(uu, u0, dt), u0)
        out.append(u.value())
        if on_step:
            on_step(u)
        u0 = u
    return out


def two_phase(er, perm, poro, watervisc, oilvisc, source_cells, source_values, sw_initial, timesteps,
              anchor_cells, corey=1.0, on_step=None):
    """Fully implicit two-phase flow; returns [(p, sw)] after each step.

    With rate-controlled wells only, incompressible pressure is defined up to
    a constant; the pressure equation of the `anchor_cells` is replaced by
    p = 0 there (their mass balance follows from the others').  The Newton
    guess for Sw is the previous step's saturation."""
    pv = er.collection(poro) * er.norm(er.allCells())

    def compute_trans(permeability):
        interior_faces = er.interiorFaces()
        first = er.firstCell(interior_faces)
        second = er.secondCell(interior_faces)
        cdiff1 = er.centroid(first) - er.centroid(interior_faces)
        cdiff2 = er.centroid(second) - er.centroid(interior_faces)
        p1 = er.operatorOn(permeability, er.allCells(), first)
        p2 = er.operatorOn(permeability, er.allCells(), second)
        a = er.norm(interior_faces)
        halftrans1 = (-a * p1) * (er.dot(er.normal(interior_faces), cdiff1) / er.dot(cdiff1, cdiff1))
        halftrans2 = (a * p2) * (er.dot(er.normal(interior_faces), cdiff2) / er.dot(cdiff2, cdiff2))
        return 1.0 / ((1.0 / halftrans1) + (1.0 / halftrans2))

    trans = compute_trans(er.collection(perm))

    def upwind(flux, x):
        x1 = er.operatorOn(x, er.allCells(), er.firstCell(er.interiorFaces()))
        x2 = er.operatorOn(x, er.allCells(), er.secondCell(er.interiorFaces()))
        return er.trinaryIf(flux >= 0.0, x1, x2)

    def total_flux(pressure, total_mob):
        ngradp = -er.gradient(pressure)
        face_total_mobility = upwind(ngradp, total_mob)
        return (trans * face_total_mobility) * ngradp

    def relperm(s):
        return s if corey == 1.0 else s * s

    def water_mob(sw):
        return relperm(sw) / watervisc

    def oil_mob(sw):
        so = er.operatorExtend(1.0, er.allCells()) - sw
        return relperm(so) / oilvisc

    anchor_set = er.entity_set(capi.CELLS, anchor_cells)
    is_anchor = er.operatorExtend(er.operatorExtend(1.0, anchor_set), anchor_set, er.allCells()) > 0.5

    def pressure_residual(pressure, total_mob, source, dt):
        # scaled by dt/pv like the transport residual, so both rows are in
        # units of saturation
        balance = (dt / pv) * (er.divergence(total_flux(pressure, total_mob)) - source)
        return er.trinaryIf(is_anchor, pressure, balance)

    def transport_residual(sw, sw0, flux, source, insource_sw, dt):
        insource = er.trinaryIf(source > 0.0, source, er.operatorExtend(0.0, er.allCells()))
        outsource = er.trinaryIf(source < 0.0, source, er.operatorExtend(0.0, er.allCells()))
        mw = water_mob(sw)
        mo = oil_mob(sw)
        fracflow = mw / (mw + mo)
        face_fracflow = upwind(flux, fracflow)
        water_flux = face_fracflow * flux
        q = (insource * insource_sw) + (outsource * fracflow)
        return (sw - sw0) + ((dt / pv) * (er.divergence(water_flux) - q))

    src_cells = er.entity_set(capi.CELLS, source_cells)
    source = er.operatorExtend(er.collection(source_values), src_cells, er.allCells())
    insource_sw = er.operatorExtend(1.0, er.allCells())
    sw0 = er.collection(sw_initial)
    p0 = er.operatorExtend(0.0, er.allCells())
    out = []
    for dt in timesteps:
        def pres(p, sw, dt=dt):
            return pressure_residual(p, water_mob(sw) + oil_mob(sw), source, dt)

        def trans_res(p, sw, sw0=sw0, dt=dt):
            flux = total_flux(p, water_mob(sw) + oil_mob(sw))
            return transport_residual(sw, sw0, flux, source, insource_sw, dt)

        p0, sw0 = er.newtonSolveSystem([pres, trans_res], [p0, sw0])
        out.append((p0.value(), sw0.value()))
        if on_step:
            on_step(p0, sw0)
    return out


# ---- seeded inputs -----------------------------------------------------------
def heat_case(nx, ny, steps=20, dt=0.5, seed=0):
    """The implicit heat-equation configuration: u0 ~ U[0.5, 1.5] per cell,
    Dirichlet u = 0.5 on the left boundary x-faces, zero flux elsewhere."""
    rng = np.random.default_rng(seed)
    u0 = rng.uniform(0.5, 1.5, nx * ny)
    dir_faces = np.array([(nx + 1) * j for j in range(ny)], dtype=np.int32)
    grid = dict(grid_dim=2, nx=nx, ny=ny, dx=1.0, dy=1.0)
    case = dict(u_initial=u0, dir_faces=dir_faces, dir_val=np.full(ny, 0.5), timesteps=[dt] * steps)
    return grid, case


def lognormal_field(shape, corr_len, std, mean_log, seed):
    """Gaussian random field with exponential covariance exp(-r/corr_len),
    std `std`, mean `mean_log`, by circulant embedding on a doubled periodic
    grid (FFT); returns exp(field), flattened with x fastest."""
    rng = np.random.default_rng(seed)
    ext = [2 * s for s in shape]
    axes = [np.minimum(np.arange(e), e - np.arange(e)) for e in ext]
    grids = np.meshgrid(*axes, indexing="ij")
    r = np.sqrt(sum(g.astype(np.float64) ** 2 for g in grids))
    cov = np.exp(-r / corr_len)
    lam = np.maximum(np.real(np.fft.fftn(cov)), 0.0)
    noise = rng.standard_normal(ext) + 1j * rng.standard_normal(ext)
    field = np.real(np.fft.ifftn(np.sqrt(lam) * noise)) * np.sqrt(np.prod(ext))
    field = field[tuple(slice(0, s) for s in shape)]
    field = (field - field.mean()) / (field.std() + 1e-300) * std + mean_log
    # shape is (nx, ny[, nz]); flatten with x fastest
    return np.exp(field).transpose().reshape(-1)


def two_phase_case(nx, ny, nz=None, steps=2, dt=86400.0, seed=0, corr_len=8.0, corey=2.0, well_pv_per_day=1.0):
    """Oil-water case: log-permeability GRF (mean ln(100 mD), std 1), porosity
    0.2, viscosities 1 cP and 5 cP, injector column in cell (0,0,*) and
    producer column in the opposite corner, Sw0 = 0.2.  Each well cell
    passes `well_pv_per_day` of its own pore volume per day (the rate
    control); dx = dy = 10 m, dz = 2 m (3D) or unit thickness (2D)."""
    shape = (nx, ny) if nz is None else (nx, ny, nz)
    mD = 9.869233e-16
    perm = lognormal_field(shape, corr_len, 1.0, np.log(100 * mD), seed)
    n = int(np.prod(shape))
    poro = np.full(n, 0.2)
    layers = 1 if nz is None else nz
    inj = [0 + nx * (0 + ny * k) for k in range(layers)]
    prod = [(nx - 1) + nx * ((ny - 1) + ny * k) for k in range(layers)]
    cells = np.array(sorted(inj + prod), dtype=np.int32)
    dz = 2.0 if nz is not None else 1.0
    per = well_pv_per_day * 0.2 * 10.0 * 10.0 * dz / 86400.0
    vals = np.array([per if c in inj else -per for c in cells], dtype=np.float64)
    grid = dict(grid_dim=2 if nz is None else 3, nx=nx, ny=ny, dx=10.0, dy=10.0)
    if nz is not None:
        grid.update(nz=nz, dz=2.0)
    case = dict(perm=perm, poro=poro, watervisc=1e-3, oilvisc=5e-3, source_cells=cells, source_values=vals,
                sw_initial=np.full(n, 0.2), timesteps=[dt] * steps, corey=corey,
                anchor_cells=np.array([prod[0]], dtype=np.int32))
    return grid, case


def swe(er, h_init, u_init, v_init, b_north, b_south, b_east, b_west, dx, dy, cfl, num_steps, on_step=None,
        heun_weight=0.5):
    """Explicit shallow-water equations (equelle_b200/sims/swe.cpp, op for
    op): Rusanov fluxes, wall fluxes, bathymetry source, Heun steps with the
    CFL time step.  Returns [(w, hu, hv)] after each step (host arrays).
    heun_weight: the weights of the final average (0.5: Heun's method;
    another value makes a different program, for tests)."""
    col = er.collection
    b_north, b_south, b_east, b_west = col(b_north), col(b_south), col(b_east), col(b_west)
    h_init, u_init, v_init = col(h_init), col(u_init), col(v_init)
    b_mid = (((b_north + b_south) + b_east) + b_west) / 4.0
    gravity, dry, dummy = 9.81, 0.05, 1000.0
    int_faces = er.interiorFaces()
    bound = er.boundaryFaces()
    cells = er.allCells()
    vol = er.norm(cells)
    area = er.norm(er.allFaces())
    int_orientation = er.normal(int_faces)
    nx, ny = int_orientation.col(0), int_orientation.col(1)
    first = er.firstCell(int_faces)
    second = er.secondCell(int_faces)
    bFirst = er.operatorOn(b_mid, cells, first)
    bSecond = er.operatorOn(b_mid, cells, second)
    bound_orientation = er.normal(bound)
    bound_cells = er.trinaryIf(er.isEmpty(er.firstCell(bound)), er.secondCell(bound), er.firstCell(bound))
    bound_b = er.operatorOn(b_mid, cells, bound_cells)
    bound_signX = er.trinaryIf(bound_orientation.col(0) > 0.0, er.operatorExtend(1.0, bound), er.operatorExtend(-1.0, bound))
    bound_signY = er.trinaryIf(bound_orientation.col(1) > 0.0, er.operatorExtend(1.0, bound), er.operatorExtend(-1.0, bound))
    bx = (b_east - b_west) / dx
    by = (b_north - b_south) / dy

    def sideFlux(w, hu, hv, b):
        rawHeight = w - b
        wet = rawHeight > dry
        height = er.trinaryIf(wet, rawHeight, er.operatorExtend(dummy, int_faces))
        qn = (hu * nx) + (hv * ny)
        un = qn / height
        pressure = (0.5 * gravity) * (height * height)
        zero = er.operatorExtend(0.0, int_faces)
        f0 = er.trinaryIf(wet, qn, zero)
        f1 = er.trinaryIf(wet, (hu * un) + (pressure * nx), zero)
        f2 = er.trinaryIf(wet, (hv * un) + (pressure * ny), zero)
        speed = er.trinaryIf(wet, er.sqrt(un * un) + er.sqrt(gravity * height), zero)
        return f0, f1, f2, speed

    def getFlux(w, hu, hv):
        wL = er.operatorOn(w, cells, first)
        huL = er.operatorOn(hu, cells, first)
        hvL = er.operatorOn(hv, cells, first)
        wR = er.operatorOn(w, cells, second)
        huR = er.operatorOn(hu, cells, second)
        hvR = er.operatorOn(hv, cells, second)
        fL = sideFlux(wL, huL, hvL, bFirst)
        fR = sideFlux(wR, huR, hvR, bSecond)
        a = er.trinaryIf(fL[3] > fR[3], fL[3], fR[3])
        intFlux0 = (0.5 * (fL[0] + fR[0])) - ((0.5 * a) * (wR - wL))
        intFlux1 = (0.5 * (fL[1] + fR[1])) - ((0.5 * a) * (huR - huL))
        intFlux2 = (0.5 * (fL[2] + fR[2])) - ((0.5 * a) * (hvR - hvL))
        bound_height = er.operatorOn(w, cells, bound_cells) - bound_b
        b_flux = er.trinaryIf(bound_height > dry, (0.5 * gravity) * (bound_height * bound_height),
                              er.operatorExtend(0.0, bound))
        boundFlux1 = (er.sqrt(bound_orientation.col(0) * bound_orientation.col(0)) * b_flux) * bound_signX
        boundFlux2 = (er.sqrt(bound_orientation.col(1) * bound_orientation.col(1)) * b_flux) * bound_signY
        all_faces = er.allFaces()
        all0 = er.operatorExtend(intFlux0, int_faces, all_faces) * area
        all1 = (er.operatorExtend(intFlux1, int_faces, all_faces) + er.operatorExtend(boundFlux1, bound, all_faces)) * area
        all2 = (er.operatorExtend(intFlux2, int_faces, all_faces) + er.operatorExtend(boundFlux2, bound, all_faces)) * area
        return all0, all1, all2

    def sourceTerm(w):
        secondTerm_x = ((w - b_east) + (w - b_west)) / 2.0
        secondTerm_y = ((w - b_north) + (w - b_south)) / 2.0
        dryTerm = er.trinaryIf((w - b_mid) > dry, er.operatorExtend(1.0, cells), er.operatorExtend(0.0, cells))
        return (((-gravity) * bx) * secondTerm_x) * dryTerm, (((-gravity) * by) * secondTerm_y) * dryTerm

    def eulerStage(w, hu, hv, dt):
        flux = getFlux(w, hu, hv)
        source = sourceTerm(w)
        w1 = w + ((dt / vol) * (-er.divergence(flux[0])))
        hu1 = hu + ((dt / vol) * ((-er.divergence(flux[1])) + (vol * source[0])))
        hv1 = hv + ((dt / vol) * ((-er.divergence(flux[2])) + (vol * source[1])))
        return w1, hu1, hv1

    def maxSpeed(w, hu, hv):
        rawHeight = w - b_mid
        wet = rawHeight > dry
        height = er.trinaryIf(wet, rawHeight, er.operatorExtend(dummy, cells))
        u = hu / height
        v = hv / height
        speed = er.trinaryIf(wet, er.sqrt((u * u) + (v * v)) + er.sqrt(gravity * height), er.operatorExtend(0.0, cells))
        return er.maxReduce(speed)

    w0 = h_init + b_mid
    hu0 = h_init * u_init
    hv0 = h_init * v_init
    h_min = dx if dx < dy else dy
    out = []
    for _ in range(int(num_steps)):
        dt = (cfl * h_min) / maxSpeed(w0, hu0, hv0)
        qs = eulerStage(w0, hu0, hv0, dt)
        qss = eulerStage(qs[0], qs[1], qs[2], dt)
        w0 = (heun_weight * w0) + (heun_weight * qss[0])
        hu0 = (heun_weight * hu0) + (heun_weight * qss[1])
        hv0 = (heun_weight * hv0) + (heun_weight * qss[2])
        out.append((w0.value(), hu0.value(), hv0.value()))
        if on_step:
            on_step(w0, hu0, hv0)
    return out


def swe_case(nx, ny, steps=200, seed=0, bumps=8, amplitude=0.1, sigma=40.0, bottom=0.05, dx=1.0, dy=1.0):
    """Dam-break-like shallow-water case: depth 1 plus `bumps` Gaussian
    bumps (amplitude, sigma in cells, centres uniform over the domain), zero
    momentum, bottom b = bottom * sin(2 pi kx x / Lx + px) sin(2 pi ky y / Ly
    + py) with kx, ky in {1..4} and phases from the seed, evaluated at the
    cell faces' midpoints.  Returns (grid parameters, swe() keyword
    arguments)."""
    rng = np.random.default_rng(seed)
    xc = (np.arange(nx) + 0.5) * dx
    yc = (np.arange(ny) + 0.5) * dy
    X, Y = np.meshgrid(xc, yc)  # [j, i]: cell i + nx j
    h = np.ones((ny, nx))
    cx = rng.uniform(0.0, nx * dx, bumps)
    cy = rng.uniform(0.0, ny * dy, bumps)
    for k in range(bumps):
        r2 = (X - cx[k]) ** 2 + (Y - cy[k]) ** 2
        h += amplitude * np.exp(-r2 / (2.0 * (sigma * dx) ** 2))
    kx, ky = rng.integers(1, 5, 2)
    px, py = rng.uniform(0.0, 2.0 * np.pi, 2)
    Lx, Ly = nx * dx, ny * dy

    def b(x, y):
        return bottom * np.sin(2.0 * np.pi * kx * x / Lx + px) * np.sin(2.0 * np.pi * ky * y / Ly + py)

    n = nx * ny
    flat = lambda a: np.ascontiguousarray(a.reshape(n))
    grid = dict(grid_dim=2, nx=nx, ny=ny, dx=dx, dy=dy)
    case = dict(h_init=flat(h), u_init=np.zeros(n), v_init=np.zeros(n),
                b_north=flat(b(X, Y + 0.5 * dy)), b_south=flat(b(X, Y - 0.5 * dy)),
                b_east=flat(b(X + 0.5 * dx, Y)), b_west=flat(b(X - 0.5 * dx, Y)),
                dx=dx, dy=dy, cfl=0.45, num_steps=steps)
    return grid, case
