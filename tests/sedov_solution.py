"""Self-similar Sedov-Taylor blast wave (point explosion in a uniform gas at rest).

Test infrastructure: the analytic reference of the Sedov tests (the reference checks its
numerical blast against numtools/sedov.f90 in tests/sedov3d.f90:123-127 and
tests/sedov2d.f90).  Restated here from the published similarity formulation (Sedov 1959,
Taylor 1950), integrated numerically:

With R(t) = xi0 (E t^2 / rho0)^(1/(j+2)) the shock radius (j = 3 spherical, 2 cylindrical),
delta = 2/(j+2) (so dR/dt = delta R / t), lambda = r / R and the ansatz
    rho = rho0 G(lambda),  u = dR/dt U(lambda),  p = rho0 (dR/dt)^2 P(lambda),
the Euler equations (continuity, momentum, entropy p rho^-gamma conserved along paths) become
    (U - l) G' + G U'                    = -(j - 1) G U / l
    (U - l) U' + P' / G                  = -(delta - 1) / delta U
    (U - l) P' / P - gamma (U - l) G'/G  = -2 (delta - 1) / delta
with the strong-shock conditions at l = 1: U = P = 2/(gamma+1), G = (gamma+1)/(gamma-1).
The profiles are integrated from the shock inwards; the total energy
    E = A_j rho0 (dR/dt)^2 R^j integral_0^1 (G U^2 / 2 + P / (gamma - 1)) l^(j-1) dl,
A_3 = 4 pi, A_2 = 2 pi, fixes xi0^(j+2) = 1 / (A_j delta^2 I).  Published values of xi0
(gamma = 1.4: 1.033 spherical; gamma = 5/3: 1.152 spherical) check the integration.
"""
import numpy as np
from scipy.integrate import solve_ivp


class Sedov:
    def __init__(self, j=3, gamma=1.4, rho0=1.0, energy=1.0, p0=0.0, lmin=1e-5):
        self.j, self.gamma, self.rho0, self.energy, self.p0 = j, gamma, rho0, energy, p0
        g = gamma
        self.delta = 2.0 / (j + 2)
        dl = self.delta

        def rhs(lam, y):
            G, U, P = y
            w = U - lam
            # A x = b for x = (G', U', P')
            A = np.array([[w, G, 0.0],
                          [0.0, w, 1.0 / G],
                          [-g * w / G, 0.0, w / P]])
            b = np.array([-(j - 1) * G * U / lam, -(dl - 1.0) / dl * U, -2.0 * (dl - 1.0) / dl])
            return np.linalg.solve(A, b)

        y1 = [(g + 1.0) / (g - 1.0), 2.0 / (g + 1.0), 2.0 / (g + 1.0)]
        sol = solve_ivp(rhs, (1.0, lmin), y1, method="LSODA", rtol=1e-11, atol=1e-14, dense_output=True)
        if not sol.success:
            raise RuntimeError("Sedov profile integration failed: " + sol.message)
        lam = np.linspace(1.0, lmin, 20001)
        G, U, P = sol.sol(lam)
        area = 4.0 * np.pi if j == 3 else 2.0 * np.pi
        f = (0.5 * G * U ** 2 + P / (g - 1.0)) * lam ** (j - 1)
        # trapezoidal rule on the fine grid (the integrand is smooth and vanishes at 0)
        I = float(np.sum(0.5 * (f[1:] + f[:-1]) * (lam[:-1] - lam[1:])))
        self.xi0 = (1.0 / (area * dl ** 2 * I)) ** (1.0 / (j + 2))
        self._sol = sol
        self.lmin = lmin

    def radius(self, t):
        return self.xi0 * (self.energy * t * t / self.rho0) ** (1.0 / (self.j + 2))

    def time_of_radius(self, r):
        """Time at which the shock reaches radius r."""
        return np.sqrt(self.rho0 / self.energy * (r / self.xi0) ** (self.j + 2))

    def state(self, r, t):
        """(density, radial velocity, pressure) at radii r (array) and time t."""
        r = np.asarray(r, dtype=np.float64)
        R = self.radius(t)
        Rdot = self.delta * R / t
        lam = np.clip(r / R, self.lmin, 1.0)
        G, U, P = self._sol.sol(lam.ravel())
        G, U, P = G.reshape(r.shape), U.reshape(r.shape), P.reshape(r.shape)
        inside = r <= R
        rho = np.where(inside, self.rho0 * G, self.rho0)
        vel = np.where(inside, Rdot * U, 0.0)
        pre = np.where(inside, np.maximum(self.rho0 * Rdot ** 2 * P, self.p0), self.p0)
        return rho, vel, pre
