"""FFT Green's-function half-spaces on the B200.

Drop-in for ``PeriodicFFTElasticHalfSpace`` and ``FreeFFTElasticHalfSpace``
of ContactMechanics/FFTElasticHalfSpace.py (v1.8.3).  The constructor
arguments, properties, ``evaluate_disp`` / ``evaluate_force`` semantics and
errors follow the reference; the transforms, Green's tables and the
multiply run in ``libcm_b200.so`` (hand-written sm_100a kernels).

Arrays: numpy arrays are copied to the device and results come back as
numpy arrays (the reference returns new arrays too); torch CUDA tensors are
used in place and results are returned as torch CUDA tensors.
"""
import ctypes

import numpy as np

from . import _lib
from .Substrates import ElasticSubstrate


def _torch():
    import torch
    return torch


def _host(a):
    if hasattr(a, "detach") and hasattr(a, "cpu"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


class _Plan:
    """Owns one ``cm_plan`` (device tables, twiddles, work buffers)."""

    def __init__(self, desc):
        L = _lib.lib()
        self._L = L
        # the launch shapes the package's autotuner measured for this GPU
        from .Autotune import apply_default
        apply_default()
        ptr = ctypes.c_void_p()
        _lib.check(L.cm_plan_create(ctypes.byref(desc), None, ctypes.byref(ptr)))
        self.ptr = ptr
        nxd, nyd, nyh = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(L.cm_plan_shape(ptr, ctypes.byref(nxd), ctypes.byref(nyd), ctypes.byref(nyh)))
        self.domain = (nxd.value, nyd.value)
        self.nyh = nyh.value

    def greens_table(self):
        out = np.empty((self.domain[0], self.nyh), dtype=np.float64)
        _lib.check(self._L.cm_plan_greens_host(self.ptr, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def __del__(self):
        try:
            if self.ptr:
                self._L.cm_plan_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass


class PeriodicFFTElasticHalfSpace(ElasticSubstrate):
    """Periodic elastic half-space (FFTElasticHalfSpace.py:151-885).

    Extra keyword ``precision`` ("fp64" default, or "fp32") selects the
    arithmetic of ``evaluate_disp`` / ``evaluate_force``; the solver picks
    its own precision.
    """

    name = "periodic_fft_elastic_halfspace"
    _periodic = True

    def __init__(self, nb_grid_pts, young, physical_sizes=2 * np.pi, stiffness_q0=None,
                 thickness=None, poisson=0.0, superclass=True, fft="serial",
                 communicator=None, fftengine=None, precision="fp64"):
        super().__init__()
        if not hasattr(nb_grid_pts, "__iter__"):
            nb_grid_pts = (nb_grid_pts,)
        if not hasattr(physical_sizes, "__iter__"):
            physical_sizes = (physical_sizes,)
        self.__dim = len(nb_grid_pts)
        if self.dim not in (1, 2):
            raise self.Error(
                ("Dimension of this problem is {}. Only 1 and 2-dimensional "
                 "problems are supported").format(self.dim))
        if stiffness_q0 is not None and thickness is not None:
            raise self.Error("Please specify either stiffness_q0 or thickness or neither.")
        self._nb_grid_pts = tuple(int(n) for n in nb_grid_pts)
        self._physical_sizes = tuple(
            physical_sizes[min(i, len(physical_sizes) - 1)] for i in range(self.dim))
        self._steps = tuple(float(size) / res for size, res in
                            zip(self.physical_sizes, self.nb_grid_pts))
        self.young = young
        self.poisson = poisson
        self.contact_modulus = young / (1 - poisson ** 2)
        self.stiffness_q0 = stiffness_q0
        self.thickness = thickness
        self._communicator = communicator
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        self.precision = precision
        self._greens = None
        self._plan = None
        if superclass:
            self._plan = _Plan(self._plan_desc())

    # --- plan description -------------------------------------------------
    def _plan_desc(self):
        d = _lib.PlanDesc()
        d.kind = _lib.CM_PERIODIC
        d.dim = self.dim
        d.nx = self.nb_grid_pts[0]
        d.ny = self.nb_grid_pts[1] if self.dim == 2 else 1
        d.sx = float(self.physical_sizes[0])
        d.sy = float(self.physical_sizes[1]) if self.dim == 2 else 1.0
        d.young = float(self.young)
        d.poisson = float(self.poisson)
        if self.stiffness_q0 is None:
            d.q0_mode = _lib.CM_Q0_DEFAULT
        elif self.stiffness_q0 == 0.0:
            d.q0_mode = _lib.CM_Q0_ZERO
        else:
            d.q0_mode = _lib.CM_Q0_VALUE
            d.stiffness_q0 = float(self.stiffness_q0)
        d.thickness = float(self.thickness) if self.thickness is not None else 0.0
        return d

    # --- geometry (FFTElasticHalfSpace.py:308-430) --------------------------
    @property
    def dim(self):
        return self.__dim

    @property
    def nb_grid_pts(self):
        return self._nb_grid_pts

    @property
    def area_per_pt(self):
        return np.prod(self.physical_sizes) / np.prod(self.nb_grid_pts)

    @property
    def physical_sizes(self):
        return self._physical_sizes

    @property
    def nb_domain_grid_pts(self):
        return self.nb_grid_pts

    @property
    def nb_subdomain_grid_pts(self):
        return self.nb_domain_grid_pts

    @property
    def topography_nb_subdomain_grid_pts(self):
        return self.nb_subdomain_grid_pts

    @property
    def subdomain_locations(self):
        return (0,) * self.dim

    @property
    def topography_subdomain_locations(self):
        return self.subdomain_locations

    @property
    def subdomain_slices(self):
        return tuple(slice(s, s + n) for s, n in
                     zip(self.subdomain_locations, self.nb_subdomain_grid_pts))

    @property
    def topography_subdomain_slices(self):
        return tuple(slice(s, s + n) for s, n in
                     zip(self.topography_subdomain_locations,
                         self.topography_nb_subdomain_grid_pts))

    @property
    def local_topography_subdomain_slices(self):
        return tuple(slice(0, n) for n in self.topography_nb_subdomain_grid_pts)

    @property
    def nb_fourier_grid_pts(self):
        d = self.nb_domain_grid_pts
        return (d[0] // 2 + 1,) + tuple(d[1:])

    @property
    def fourier_locations(self):
        return (0,) * self.dim

    @property
    def fourier_slices(self):
        return tuple(slice(0, n) for n in self.nb_fourier_grid_pts)

    @property
    def communicator(self):
        return self._communicator

    def __repr__(self):
        dims = "x", "y", "z"
        size_str = ", ".join("{}: {}({})".format(d, s, n) for d, s, n in
                             zip(dims, self.physical_sizes, self.nb_grid_pts))
        return ("{0.dim}-dimensional halfspace '{0.name}', "
                "physical_sizes(nb_grid_pts) in {1}, E' = {0.young}".format(self, size_str))

    # --- Green's tables (:445-571) -----------------------------------------
    @property
    def greens_function(self):
        """Green's table in the reference layout: complex, halved along x."""
        if self._greens is None:
            g = self._plan.greens_table()           # (nxd, nyh), halved along y
            nxd, nyd = self._plan.domain
            if self.dim == 1:
                ref = g[:nxd // 2 + 1, 0]
            else:
                ky = np.arange(nyd)
                ref = g[:nxd // 2 + 1, np.minimum(ky, nyd - ky)]
            self._greens = ref.astype(complex)
        return self._greens

    @property
    def surface_stiffness(self):
        g = self.greens_function
        k = np.zeros(g.shape, dtype=complex)
        k[g != 0] = 1.0 / g[g != 0]
        return k

    # --- operators (:573-611) ----------------------------------------------
    def _apply(self, op, field, out_shape, in_rows, in_cols, out_rows, out_cols, precision=None):
        torch = _torch()
        prec = precision or self.precision
        tdt = torch.float64 if prec == "fp64" else torch.float32
        is_np = not isinstance(field, torch.Tensor)
        if is_np:
            src = torch.from_numpy(np.ascontiguousarray(field, dtype=np.float64)).to(
                device="cuda", dtype=tdt)
        else:
            src = field.to(dtype=tdt).contiguous()
            if not src.is_cuda:
                src = src.cuda()
        if self.dim == 1:
            src = src.reshape(-1, 1)
        out = torch.empty((out_rows, out_cols), dtype=tdt, device="cuda")
        L = self._plan._L
        # torch's default stream has the handle 0, which the library reads as
        # "the plan's stream"; name the legacy default stream explicitly
        stream = torch.cuda.current_stream().cuda_stream or _lib.CUDA_STREAM_LEGACY
        _lib.check(L.cm_apply(self._plan.ptr, op, _lib.PRECISIONS[prec],
                              ctypes.c_void_p(src.data_ptr()), in_rows, in_cols, src.shape[1],
                              ctypes.c_void_p(out.data_ptr()), out_rows, out_cols, out_cols,
                              ctypes.c_void_p(stream)))
        out = out.reshape(out_shape)
        if is_np:
            return out.to(torch.float64).cpu().numpy()
        return out

    def _shape(self, a):
        return tuple(a.shape)

    def evaluate_disp(self, forces):
        """Displacements due to point forces (FFTElasticHalfSpace.py:573-589)."""
        if self._shape(forces) != self.nb_subdomain_grid_pts:
            raise self.Error(
                ("force array has a different shape ({0}) than this halfspace's "
                 "nb_grid_pts ({1})").format(self._shape(forces), self.nb_subdomain_grid_pts))
        nxd = self.nb_domain_grid_pts[0]
        nyd = self.nb_domain_grid_pts[1] if self.dim == 2 else 1
        return self._apply(_lib.CM_OP_DISP, forces, self.nb_domain_grid_pts, nxd, nyd, nxd, nyd)

    def evaluate_force(self, disp):
        """Point forces due to a displacement field (FFTElasticHalfSpace.py:591-611)."""
        if self._shape(disp) != self.nb_subdomain_grid_pts:
            raise self.Error(
                ("displacements array has a different shape ({0}) than this halfspace's "
                 "nb_grid_pts ({1})").format(self._shape(disp), self.nb_subdomain_grid_pts))
        nxd = self.nb_domain_grid_pts[0]
        nyd = self.nb_domain_grid_pts[1] if self.dim == 2 else 1
        return self._apply(_lib.CM_OP_FORCE, disp, self.nb_domain_grid_pts, nxd, nyd, nxd, nyd)

    def evaluate_elastic_energy(self, forces, disp):
        """``0.5 * dot(disp, -forces)`` (FFTElasticHalfSpace.py:676-684)."""
        return 0.5 * float(np.dot(np.ravel(_host(disp)), np.ravel(-_host(forces))))

    # --- k-space (:613-805, 841-885): half spectra in the reference's
    # layout, complex (nxd // 2 + 1, nyd), halved along x, unnormalised ----
    def _kshape(self):
        return self.nb_fourier_grid_pts

    def _k_device(self, a):
        """A contiguous complex128 device copy (or view) of a half spectrum."""
        torch = _torch()
        if isinstance(a, torch.Tensor):
            t = a.to(device="cuda", dtype=torch.complex128).contiguous()
        else:
            t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.complex128)).cuda()
        if tuple(t.shape) != self._kshape():
            raise self.Error("Fourier array has shape {} but this halfspace's half spectrum "
                             "has shape {}".format(tuple(t.shape), self._kshape()))
        return t

    def _fft(self, field):
        """Forward transform of a domain-shaped real field (device FP64)."""
        torch = _torch()
        is_np = not isinstance(field, torch.Tensor)
        src = (torch.from_numpy(np.ascontiguousarray(field, dtype=np.float64)).cuda() if is_np
               else field.to(device="cuda", dtype=torch.float64).contiguous())
        nxd = self.nb_domain_grid_pts[0]
        nyd = self.nb_domain_grid_pts[1] if self.dim == 2 else 1
        src = src.reshape(nxd, nyd)
        out = torch.empty(self._kshape(), dtype=torch.complex128, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream or _lib.CUDA_STREAM_LEGACY
        _lib.check(self._plan._L.cm_fft_forward(self._plan.ptr, ctypes.c_void_p(src.data_ptr()),
                                                nxd, nyd, nyd, ctypes.c_void_p(out.data_ptr()),
                                                ctypes.c_void_p(stream)))
        return out, is_np

    def _kapply(self, op, scale, k, as_numpy):
        torch = _torch()
        out = torch.empty_like(k)
        stream = torch.cuda.current_stream().cuda_stream or _lib.CUDA_STREAM_LEGACY
        _lib.check(self._plan._L.cm_kspace_apply(self._plan.ptr, op, float(scale),
                                                 ctypes.c_void_p(k.data_ptr()),
                                                 ctypes.c_void_p(out.data_ptr()),
                                                 ctypes.c_void_p(stream)))
        return out.cpu().numpy() if as_numpy else out

    def evaluate_k_disp(self, forces):
        """k-space displacements ``G fft(-f) / a`` (FFTElasticHalfSpace.py:613-636)."""
        if self._shape(forces) != self.nb_subdomain_grid_pts:
            raise self.Error(
                ("force array has a different shape ({0}) than this halfspace's "
                 "nb_grid_pts ({1})").format(self._shape(forces), self.nb_subdomain_grid_pts))
        k, is_np = self._fft(forces)
        return self._kapply(_lib.CM_OP_DISP, -1.0 / self.area_per_pt, k, is_np)

    def evaluate_k_force(self, disp):
        """k-space forces ``-K fft(u) a`` (FFTElasticHalfSpace.py:638-655)."""
        if self._shape(disp) != self.nb_subdomain_grid_pts:
            raise self.Error(
                ("displacements array has a different shape ({0}) than this halfspace's "
                 "nb_grid_pts ({1})").format(self._shape(disp), self.nb_subdomain_grid_pts))
        k, is_np = self._fft(disp)
        return self._kapply(_lib.CM_OP_FORCE, -self.area_per_pt, k, is_np)

    def evaluate_k_force_k(self, disp_k):
        """k-space forces of k-space displacements ``-K u_k a`` (:657-674)."""
        torch = _torch()
        as_np = not isinstance(disp_k, torch.Tensor)
        return self._kapply(_lib.CM_OP_FORCE, -self.area_per_pt, self._k_device(disp_k), as_np)

    def evaluate_scalar_product_k_space(self, ka, kb):
        """sum_ij a_ij b_ij from the half spectra of a and b (power theorem,
        FFTElasticHalfSpace.py:686-805)."""
        a, b = self._k_device(ka), self._k_device(kb)
        out = ctypes.c_double()
        torch = _torch()
        stream = torch.cuda.current_stream().cuda_stream or _lib.CUDA_STREAM_LEGACY
        _lib.check(self._plan._L.cm_kspace_dot(self._plan.ptr, ctypes.c_void_p(a.data_ptr()),
                                               ctypes.c_void_p(b.data_ptr()), ctypes.byref(out),
                                               ctypes.c_void_p(stream)))
        return out.value

    def evaluate_elastic_energy_k_space(self, kforces, kdisp):
        """``-1/2 sum u f`` from half spectra (FFTElasticHalfSpace.py:807-839)."""
        return -0.5 * self.evaluate_scalar_product_k_space(kdisp, kforces)

    def evaluate(self, disp, pot=True, forces=False):
        """Energy and/or forces of a displacement field (FFTElasticHalfSpace.py:841-868):
        with forces, the energy is the real-space product; without, it is
        evaluated in k-space from the transform of the displacements."""
        force = potential = None
        if forces:
            force = self.evaluate_force(disp)
            if pot:
                potential = self.evaluate_elastic_energy(force, disp)
        elif pot:
            dispk, _ = self._fft(disp)
            kforce = self._kapply(_lib.CM_OP_FORCE, -self.area_per_pt, dispk, False)
            potential = self.evaluate_elastic_energy_k_space(kforce, dispk)
        return potential, force

    def evaluate_k(self, disp_k, pot=True, forces=False):
        """Energy and k-space forces of a k-space displacement field (:870-885);
        like the reference, the forces come back whenever either is asked for."""
        if not (pot or forces):
            return None, None
        force_k = self.evaluate_k_force_k(disp_k)
        potential = self.evaluate_elastic_energy_k_space(force_k, disp_k) if pot else None
        return potential, force_k


class FreeFFTElasticHalfSpace(PeriodicFFTElasticHalfSpace):
    """Non-periodic half-space with Hockney padding (FFTElasticHalfSpace.py:888-1283)."""

    name = "free_fft_elastic_halfspace"
    _periodic = False

    def __init__(self, nb_grid_pts, young, physical_sizes=2 * np.pi, fft="serial",
                 communicator=None, check_boundaries=False, fftengine=None, precision="fp64"):
        if not hasattr(nb_grid_pts, "__iter__"):
            nb_grid_pts = (nb_grid_pts,)
        self._comp_nb_grid_pts = self._domain_of(tuple(int(r) for r in nb_grid_pts))
        super().__init__(nb_grid_pts, young, physical_sizes, superclass=False, fft=fft,
                         communicator=communicator, fftengine=fftengine, precision=precision)
        if self.dim != 2:
            raise self.Error("FreeFFTElasticHalfSpace is implemented for 2D only")
        self._plan = _Plan(self._plan_desc())
        self._check_boundaries = check_boundaries

    def _domain_of(self, nb_grid_pts):
        """Computational grid: doubled along every axis (:950-951)."""
        return tuple(2 * n for n in nb_grid_pts)

    def _plan_desc(self):
        d = super()._plan_desc()
        d.kind = _lib.CM_FREE
        d.poisson = 0.0
        d.q0_mode = _lib.CM_Q0_DEFAULT
        d.thickness = 0.0
        return d

    def spawn_child(self, nb_grid_pts):
        size = tuple(nb_grid_pts[i] / float(self.nb_grid_pts[i]) * self.physical_sizes[i]
                     for i in range(self.dim))
        return type(self)(nb_grid_pts, self.young, size)

    @property
    def nb_domain_grid_pts(self):
        return self._comp_nb_grid_pts

    @property
    def topography_nb_subdomain_grid_pts(self):
        return tuple(max(0, min(self.nb_grid_pts[i] - self.subdomain_locations[i],
                                self.nb_subdomain_grid_pts[i])) for i in range(self.dim))

    @property
    def domain_boundary_mask(self):
        """Points on the boundary of the topography domain (:992-1023)."""
        mask = np.zeros(self.topography_nb_subdomain_grid_pts, dtype=bool)
        mask[:, 0] = True
        mask[:, self.nb_grid_pts[1] - 1] = True
        mask[0, :] = True
        mask[self.nb_grid_pts[0] - 1, :] = True
        return mask

    def evaluate_disp(self, forces, bIncludePadding=False):
        """Padded forces go straight through; unpadded forces are zero-padded on
        the device and only the topography quadrant is returned unless
        ``bIncludePadding`` (FFTElasticHalfSpace.py:1141-1197)."""
        shape = self._shape(forces)
        nxd, nyd = self.nb_domain_grid_pts
        if shape == self.nb_subdomain_grid_pts:
            return super().evaluate_disp(forces)
        if shape == self.nb_grid_pts:
            nx, ny = self.nb_grid_pts
            if bIncludePadding:
                return self._apply(_lib.CM_OP_DISP, forces, (nxd, nyd), nx, ny, nxd, nyd)
            return self._apply(_lib.CM_OP_DISP, forces, (nx, ny), nx, ny, nx, ny)
        raise self.Error(
            "force array has a different shape ({0}) than the subdomain nb_grid_pts ({1}), "
            "this halfspace's nb_grid_pts ({2}) or half of it.".format(
                shape, self.nb_subdomain_grid_pts, self.nb_domain_grid_pts))

    class FreeBoundaryError(Exception):
        """Forces reach the boundary of the topography domain (:1207-1215)."""

        def __init__(self, message):
            super().__init__(message)

    def check_boundaries(self, force=None, tol=0):
        """Raise if forces on the outer ring of the topography are not zero
        (FFTElasticHalfSpace.py:1217-1270)."""
        if force is None:
            force = self.force
        force = np.asarray(force)
        nx, ny = self.nb_grid_pts
        ok = (np.all(abs(force[:, 0]) <= tol) and np.all(abs(force[:, ny - 1]) <= tol)
              and np.all(abs(force[0, :]) <= tol) and np.all(abs(force[nx - 1, :]) <= tol))
        if not ok:
            raise self.FreeBoundaryError(
                "The forces not zero at the boundary of the active domain."
                "This is typically an indication that the contact geometry "
                "exceeds the bounds of the domain. Since this is a nonperiodic"
                "calculation, you may want to increase the size of your "
                "domain. If you are sure that the calculation is correct,"
                " set check_boundary to False")

    def check(self, force=None):
        if self._check_boundaries:
            self.check_boundaries(force)


class SemiPeriodicFFTElasticHalfSpace(FreeFFTElasticHalfSpace):
    """Half-space that is periodic along some axes and free along the others
    (FFTElasticHalfSpace.py:1286-1615).  A periodic axis keeps its n points
    and the Love kernel is summed over its periodic images
    -n_images..n_images; a free axis is padded to 2n - 1 points.  The kernel
    and its table are built by the library (extended-precision sum of the
    images on the host, FP64 transform on the device); evaluate_disp pads
    like FreeFFTElasticHalfSpace, evaluate_force zero-pads displacements that
    do not cover the domain."""

    name = "semi_periodic_fft_elastic_halfspace"

    def __init__(self, nb_grid_pts, young, physical_sizes=(2 * np.pi, 2 * np.pi),
                 periodicity=(False, True), n_images=10, fft="serial", communicator=None,
                 check_boundaries=False, fftengine=None, precision="fp64"):
        self.periodicity = tuple(bool(p) for p in periodicity)
        self.n_images = int(n_images)
        self._G_real = None
        super().__init__(nb_grid_pts, young, physical_sizes, fft=fft, communicator=communicator,
                         check_boundaries=check_boundaries, fftengine=fftengine,
                         precision=precision)

    def _domain_of(self, nb_grid_pts):
        """n points along a periodic axis, 2n - 1 along a free one (:1343-1353)."""
        return tuple(n if per else 2 * n - 1 for n, per in zip(nb_grid_pts, self.periodicity))

    def _plan_desc(self):
        d = super()._plan_desc()
        d.kind = _lib.CM_SEMI
        d.periodic_x = int(self.periodicity[0])
        d.periodic_y = int(self.periodicity[1])
        d.n_images = self.n_images
        return d

    def spawn_child(self, nb_grid_pts):
        size = tuple(nb_grid_pts[i] / float(self.nb_grid_pts[i]) * self.physical_sizes[i]
                     for i in range(self.dim))
        return type(self)(nb_grid_pts, self.young, size, periodicity=self.periodicity,
                          n_images=self.n_images)

    def evaluate_force(self, disp):
        """Forces due to displacements (:1541-1565); displacements that do not
        cover the domain are zero padded."""
        shape = self._shape(disp)
        nxd, nyd = self.nb_domain_grid_pts
        if shape == (nxd, nyd):
            return super().evaluate_force(disp)
        if len(shape) != 2 or shape[0] > nxd or shape[1] > nyd:
            raise self.Error("displacements array has a different shape ({0}) than this "
                             "halfspace's domain ({1})".format(shape, (nxd, nyd)))
        return self._apply(_lib.CM_OP_FORCE, disp, (nxd, nyd), shape[0], shape[1], nxd, nyd)

    @property
    def G_real(self):
        """Real-space kernel of the domain (sum over the periodic images)."""
        if self._G_real is None:
            nxd, nyd = self.nb_domain_grid_pts
            self._G_real = np.fft.irfftn(self.greens_function, s=(nyd, nxd), axes=(1, 0))
        return self._G_real

    def get_G_real(self):
        """The real-space kernel with the zero offset at the array centre (:1567-1596)."""
        nxd, nyd = self.nb_domain_grid_pts
        mx = np.round(np.fft.fftfreq(nxd) * nxd).astype(int)
        my = np.round(np.fft.fftfreq(nyd) * nyd).astype(int)
        return self.G_real[np.ix_(np.argsort(mx), np.argsort(my))]

    def get_G_real_slices(self):
        """Middle slices of get_G_real() along x and along y (:1598-1615)."""
        g = self.get_G_real()
        return g[:, g.shape[1] // 2], g[g.shape[0] // 2, :]
