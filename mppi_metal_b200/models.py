"""Parameter blobs of the shipped model plugins and the seeded workloads.

``ctypes`` mirrors of mppi_metal_b200/plugins/model_params.h, plus builders
for the benchmark problems.  No public benchmark data is involved: every
workload is drawn from numpy's PCG64 generator with a fixed seed, with the
shapes, sizes and value ranges of the configurations it stands for.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

UNICYCLE_MAX_OBS = 16
BICYCLE_MAX_SEGMENTS = 32
QUAD_MAX_OBS = 32

_f = ctypes.c_float
_u = ctypes.c_uint32


class NonholonomicModelParams(ctypes.Structure):
    _fields_ = [("v_max", _f), ("dt", _f)]


class NonholonomicCostParams(ctypes.Structure):
    _fields_ = [("x_goal", _f), ("y_goal", _f), ("goal_radius", _f), ("pos_weight", _f),
                ("heading_weight", _f), ("control_weight", _f)]


class UnicycleModelParams(ctypes.Structure):
    _fields_ = [("dt", _f), ("pad0", _f), ("pad1", _f), ("pad2", _f)]


class UnicycleCostParams(ctypes.Structure):
    _fields_ = [("goal_x", _f), ("goal_y", _f), ("w_goal", _f), ("w_obs", _f),
                ("w_terminal", _f), ("num_obs", _u), ("pad0", _f), ("pad1", _f),
                ("obs_cx", _f * UNICYCLE_MAX_OBS), ("obs_cy", _f * UNICYCLE_MAX_OBS),
                ("obs_vx", _f * UNICYCLE_MAX_OBS), ("obs_vy", _f * UNICYCLE_MAX_OBS),
                ("obs_r", _f * UNICYCLE_MAX_OBS)]


class BicycleModelParams(ctypes.Structure):
    _fields_ = [("dt", _f), ("wheelbase", _f), ("delta_max", _f), ("pad0", _f)]


class BicycleCostParams(ctypes.Structure):
    _fields_ = [("x0", _f), ("knot_dx", _f), ("num_segments", _u), ("v_ref", _f),
                ("w_lat", _f), ("w_head", _f), ("w_speed", _f), ("w_terminal", _f),
                ("coef", (_f * 4) * BICYCLE_MAX_SEGMENTS)]


class QuadrotorModelParams(ctypes.Structure):
    _fields_ = [("dt", _f), ("mass", _f), ("gravity", _f), ("arm", _f), ("yaw_coef", _f),
                ("jx", _f), ("jy", _f), ("jz", _f)]


class QuadrotorCostParams(ctypes.Structure):
    _fields_ = [("wp_x", _f), ("wp_y", _f), ("wp_z", _f), ("w_pos", _f), ("w_vel", _f),
                ("w_att", _f), ("w_rate", _f), ("w_obs", _f), ("w_terminal", _f),
                ("num_obs", _u), ("pad0", _f), ("pad1", _f),
                ("obs_cx", _f * QUAD_MAX_OBS), ("obs_cy", _f * QUAD_MAX_OBS),
                ("obs_cz", _f * QUAD_MAX_OBS), ("obs_r", _f * QUAD_MAX_OBS)]


class GustModelParams(ctypes.Structure):
    _fields_ = [("dt", _f), ("noise_std", _f), ("p_event", _f), ("gust_accel", _f)]


class WezModelParams(ctypes.Structure):
    _fields_ = [("v_max", _f), ("dt", _f), ("adv_v_max", _f), ("adv_fire_prob_max", _f),
                ("adv_max_range", _f), ("adv_min_range", _f), ("adv_k_gain", _f),
                ("adv_capture_radius", _f), ("adv_max_steps", ctypes.c_int32),
                ("num_adversaries", ctypes.c_int32)]


class WezCostParams(ctypes.Structure):
    _fields_ = [("x_goal", _f), ("y_goal", _f), ("goal_radius", _f), ("pos_weight", _f),
                ("heading_weight", _f), ("control_weight", _f), ("adv_collision_weight", _f),
                ("adv_dist_weight", _f)]


class WezAdversary(ctypes.Structure):
    _fields_ = [("x", _f), ("y", _f), ("theta", _f), ("v", _f),
                ("steps_since_active", ctypes.c_uint16), ("active", ctypes.c_bool),
                ("terminal", ctypes.c_bool)]


WEZ_ADVERSARIES = 8


class WezState(ctypes.Structure):
    """The WEZ example's AgentState: 180 bytes = 45 float slots."""
    _fields_ = [("x", _f), ("y", _f), ("theta", _f), ("v", _f), ("captured", ctypes.c_bool),
                ("adversaries", WezAdversary * WEZ_ADVERSARIES)]


WEZ_STATE_DIM = ctypes.sizeof(WezState) // 4  # 45


def blob(s: ctypes.Structure) -> bytes:
    return ctypes.string_at(ctypes.addressof(s), ctypes.sizeof(s))


@dataclass
class Workload:
    """One benchmark / parity problem, in driver terms."""
    name: str
    plugin: str
    oracle_model: str
    state_dim: int
    control_dim: int
    horizon: int
    sample_count: int
    lam: float
    sigma: np.ndarray            # shared sigma (std-devs) or covariance
    sigma_inv: np.ndarray
    u_min: np.ndarray
    u_max: np.ndarray
    num_agents: int
    num_steps: int
    x0: np.ndarray               # [N][n]
    model_params: bytes
    cost_params: list = field(default_factory=list)   # per-agent blobs
    agent_sigma: np.ndarray | None = None             # [N][m] or None
    cov_full: bool = False
    control_cost: bool = False
    seed: int = 0
    numeric_mode: int = 0  # DriverConfig::NumericMode (0 FP32, 1 FP16, 2 mixed)

    @property
    def cost_params_packed(self) -> bytes:
        return b"".join(self.cost_params)

    @property
    def cost_stride(self) -> int:
        return len(self.cost_params[0]) if self.cost_params else 0

    @property
    def rollout_steps_per_control_step(self) -> int:
        return self.num_agents * self.sample_count * self.horizon


def _unicycle_cost(rng: np.random.Generator, n_obs: int, moving: bool) -> UnicycleCostParams:
    c = UnicycleCostParams()
    gx, gy = rng.uniform(-10.0, 10.0, size=2)
    c.goal_x, c.goal_y = float(gx), float(gy)
    c.w_goal = 1.0
    c.w_obs = 1.0e3
    c.w_terminal = 10.0
    c.num_obs = n_obs
    cx = rng.uniform(-10.0, 10.0, size=n_obs)
    cy = rng.uniform(-10.0, 10.0, size=n_obs)
    r = rng.uniform(0.3, 1.0, size=n_obs)
    v = rng.uniform(-0.5, 0.5, size=(n_obs, 2)) if moving else np.zeros((n_obs, 2))
    for i in range(n_obs):
        c.obs_cx[i], c.obs_cy[i] = float(cx[i]), float(cy[i])
        c.obs_vx[i], c.obs_vy[i] = float(v[i, 0]), float(v[i, 1])
        c.obs_r[i] = float(r[i])
    return c


def unicycle_single(seed: int = 0, K: int = 1024, H: int = 30, T: int = 200) -> Workload:
    """Single-agent plain MPPI, kinematic unicycle: dt 0.05, H 30, K 1024,
    lambda 1, sigma [0.5, 0.5], v in [-1, 2], omega in [-1.5, 1.5], goal and 8
    static circles (centres U[-10,10]^2, radii U[0.3,1.0]), control cost on,
    Philox seed 0, 200 closed-loop steps from x0 = 0."""
    rng = np.random.default_rng(seed)
    mp = UnicycleModelParams(0.05, 0.0, 0.0, 0.0)
    cp = _unicycle_cost(rng, 8, moving=False)
    sigma = np.array([0.5, 0.5], np.float32)
    return Workload("unicycle_single", "unicycle_obstacles", "unicycle_obstacles", 4, 2, H, K,
                    1.0, sigma, (1.0 / sigma ** 2).astype(np.float32),
                    np.array([-1.0, -1.5], np.float32), np.array([2.0, 1.5], np.float32),
                    1, T, np.zeros((1, 4), np.float32), blob(mp), [blob(cp)], None,
                    control_cost=True, seed=seed)


def unicycle_batch(seed: int = 0, N: int = 256, K: int = 4096, H: int = 50, T: int = 300,
                   n_obs: int = 16) -> Workload:
    """Batched plain MPPI: N unicycle agents, each with its own seeded start,
    goal, 16 moving circular keep-out regions (velocities U[-0.5,0.5]^2) and
    per-dimension sigma U[0.2, 0.8]; K 4096, H 50, 300 closed-loop steps."""
    rng = np.random.default_rng(seed)
    mp = UnicycleModelParams(0.05, 0.0, 0.0, 0.0)
    x0 = np.zeros((N, 4), np.float32)
    x0[:, 0:2] = rng.uniform(-10.0, 10.0, size=(N, 2))
    x0[:, 2] = rng.uniform(-np.pi, np.pi, size=N)
    cps = [blob(_unicycle_cost(rng, n_obs, moving=True)) for _ in range(N)]
    agent_sigma = rng.uniform(0.2, 0.8, size=(N, 2)).astype(np.float32)
    sigma = np.array([0.5, 0.5], np.float32)
    return Workload("unicycle_batch", "unicycle_obstacles", "unicycle_obstacles", 4, 2, H, K,
                    1.0, sigma, (1.0 / sigma ** 2).astype(np.float32),
                    np.array([-1.0, -1.5], np.float32), np.array([2.0, 1.5], np.float32),
                    N, T, x0, blob(mp), cps, agent_sigma, control_cost=False, seed=seed)


def gust_batch(seed: int = 0, N: int = 16, K: int = 1024, H: int = 30, T: int = 20,
               lam: float = 10.0) -> Workload:
    """Stochastic dynamics (plugins/gust_integrator.cu): a double integrator
    with process noise and a random sticky gust, both drawn inside the
    dynamics from the callable's Philox counter and key; N agents start at
    rest from positions U[-3, 3]^2, sigma [1, 1], |a| <= 2, dt 0.1."""
    rng = np.random.default_rng(seed)
    mp = GustModelParams(0.1, 0.5, 0.02, 1.5)
    x0 = np.zeros((N, 5), np.float32)
    x0[:, :2] = rng.uniform(-3.0, 3.0, size=(N, 2))
    sigma = np.ones(2, np.float32)
    return Workload("gust_batch", "gust_integrator", "gust_integrator", 5, 2, H, K, lam,
                    sigma, sigma.copy(), np.full(2, -2.0, np.float32),
                    np.full(2, 2.0, np.float32), N, T, x0, blob(mp), [], None, seed=seed)


def wez_state(s: WezState) -> np.ndarray:
    """The state record as the 45 float slots the driver carries."""
    return np.frombuffer(blob(s), np.float32).copy()


def wez_fields(x: np.ndarray) -> WezState:
    """The state record behind 45 float slots."""
    return WezState.from_buffer_copy(np.ascontiguousarray(x, np.float32).tobytes())


def wez_batch(seed: int | None = None, N: int = 256, K: int = 128, H: int = 20,
              T: int = 100) -> Workload:
    """The reference's WEZ example (examples/wez_environment_batch/main.cpp:
    54-230): an ego vehicle (state x, y, theta, v, captured) driving to the
    goal (5, 5) among 8 pursuing adversaries whose engagement zones activate
    at random; K 128, H 20, lambda 1, sigma [2, 1], |a| <= 3, |omega| <= 1.5,
    dt 0.05.  Every agent starts at the origin with adversary 1 at (2, 0)
    heading pi and the others at (0, 2) heading -pi/2, all at speed 2.
    seed=None keeps the example's identical agents; a seed places each
    agent's start and goal and the adversaries at random (U[-6, 6]^2)."""
    mp = WezModelParams(2.0, 0.05, 2.0, 0.1, 8.0, 3.0, 3.0, 0.5, 100, WEZ_ADVERSARIES)
    rng = np.random.default_rng(seed) if seed is not None else None
    x0 = np.zeros((N, WEZ_STATE_DIM), np.float32)
    cps = []
    for a in range(N):
        s = WezState()
        for i in range(WEZ_ADVERSARIES):
            d = s.adversaries[i]
            d.x, d.y, d.theta = (2.0, 0.0, 3.14) if i == 0 else (0.0, 2.0, -1.57)
            d.v = 2.0
            d.steps_since_active = 0 if i == 0 else 50
        c = WezCostParams(5.0, 5.0, 0.2, 10.0, 0.0, 0.1, 100.0, 0.0)
        if rng is not None:
            s.x, s.y = (float(v) for v in rng.uniform(-6.0, 6.0, 2))
            s.theta = float(rng.uniform(-np.pi, np.pi))
            for i in range(WEZ_ADVERSARIES):
                d = s.adversaries[i]
                d.x, d.y = (float(v) for v in rng.uniform(-6.0, 6.0, 2))
                d.theta = float(rng.uniform(-np.pi, np.pi))
            c.x_goal, c.y_goal = (float(v) for v in rng.uniform(-6.0, 6.0, 2))
        x0[a] = wez_state(s)
        cps.append(blob(c))
    sigma = np.array([2.0, 1.0], np.float32)
    return Workload("wez_batch", "wez_environment", "wez_environment", WEZ_STATE_DIM, 2, H, K,
                    1.0, sigma, (1.0 / sigma).astype(np.float32),
                    np.array([-3.0, -1.5], np.float32), np.array([3.0, 1.5], np.float32), N, T,
                    x0, blob(mp), cps, None, seed=0 if seed is None else seed)


def double_integrator_test(K: int = 64, H: int = 10) -> Workload:
    """The reference test fixture (tests/mppi_driver_tests.cpp:42-72):
    n 4, m 2, H 10, K 64, lambda 1, sigma [1, 1], bounds [-1, 1]; stage cost
    px^2 + py^2 and the default (zero) terminal cost; x0 = (1, 1, 0, 0)."""
    sigma = np.ones(2, np.float32)
    return Workload("double_integrator_test", "double_integrator", "double_integrator", 4, 2, H,
                    K, 1.0, sigma, sigma.copy(), -np.ones(2, np.float32),
                    np.ones(2, np.float32), 1, 5, np.array([[1.0, 1.0, 0.0, 0.0]], np.float32),
                    b"", [], None)


def unicycle_executed_cost(states: np.ndarray, controls: np.ndarray, terminal: np.ndarray,
                           cost_blobs: list[bytes]) -> np.ndarray:
    """Closed-loop cost of executed unicycle trajectories, per agent.

    states [T][N][4] are the pre-step states, controls [T][N][2] the applied
    u*[0], terminal [N][4] the state after the last step.  The cost is the
    model's stage cost (goal distance + obstacle penetration at the model
    time) summed over the visited states x_1..x_T, plus the terminal cost of
    x_T -- what the controller actually incurred, not a sampled rollout cost.
    """
    T, N, _ = states.shape
    nxt = np.concatenate([states[1:], terminal[None]], axis=0).astype(np.float64)  # x_1..x_T
    out = np.zeros(N)
    for a in range(N):
        c = UnicycleCostParams.from_buffer_copy(cost_blobs[a])
        n_obs = min(int(c.num_obs), UNICYCLE_MAX_OBS)
        p = nxt[:, a, :]
        goal = c.w_goal * ((p[:, 0] - c.goal_x) ** 2 + (p[:, 1] - c.goal_y) ** 2)
        t = p[:, 3:4]
        cx = np.array(c.obs_cx[:n_obs]) + np.array(c.obs_vx[:n_obs]) * t
        cy = np.array(c.obs_cy[:n_obs]) + np.array(c.obs_vy[:n_obs]) * t
        d = np.sqrt((p[:, 0:1] - cx) ** 2 + (p[:, 1:2] - cy) ** 2)
        pen = np.maximum(np.array(c.obs_r[:n_obs]) - d, 0.0).sum(axis=1)
        out[a] = float(np.sum(goal + c.w_obs * pen) + c.w_terminal * goal[-1])
    return out


def natural_cubic_spline(x0: float, dx: float, ys: np.ndarray) -> np.ndarray:
    """Per-segment coefficients [c0, c1, c2, c3] (in s = x - x_i) of the
    natural cubic spline through (x0 + i dx, ys[i])."""
    n = len(ys) - 1
    a = np.zeros((n + 1, n + 1))
    rhs = np.zeros(n + 1)
    a[0, 0] = a[n, n] = 1.0
    for i in range(1, n):
        a[i, i - 1], a[i, i], a[i, i + 1] = dx, 4.0 * dx, dx
        rhs[i] = 3.0 * ((ys[i + 1] - ys[i]) - (ys[i] - ys[i - 1])) / dx
    c = np.linalg.solve(a, rhs)
    coef = np.zeros((n, 4))
    for i in range(n):
        coef[i, 0] = ys[i]
        coef[i, 1] = (ys[i + 1] - ys[i]) / dx - dx * (2.0 * c[i] + c[i + 1]) / 3.0
        coef[i, 2] = c[i]
        coef[i, 3] = (c[i + 1] - c[i]) / (3.0 * dx)
    return coef


def _random_spd(rng: np.random.Generator, lo: float, hi: float) -> np.ndarray:
    th = rng.uniform(0.0, np.pi)
    rot = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
    return rot @ np.diag(rng.uniform(lo, hi, size=2)) @ rot.T


def bicycle_uneven(seed: int = 0, N: int = 64, T: int = 100, k_range=(1024, 16384),
                   h_range=(16, 96)) -> Workload:
    """Uneven batch: N kinematic-bicycle instances (state [x,y,theta,v,delta],
    control [accel, steer_rate]) with K log-uniform in k_range and H
    log-uniform in h_range per instance, a full 2x2 noise covariance per
    instance (random SPD, eigenvalues U[0.05, 0.5]) and a lane-keeping cost on
    a seeded natural cubic-spline centreline (32 segments of 5 m)."""
    rng = np.random.default_rng(seed)
    mp = BicycleModelParams(0.05, 2.5, 0.6, 0.0)
    nseg, dx = BICYCLE_MAX_SEGMENTS, 5.0
    ys = np.cumsum(rng.uniform(-1.0, 1.0, size=nseg + 1))
    coef = natural_cubic_spline(0.0, dx, ys)
    cp = BicycleCostParams()
    cp.x0, cp.knot_dx, cp.num_segments, cp.v_ref = 0.0, dx, nseg, 5.0
    cp.w_lat, cp.w_head, cp.w_speed, cp.w_terminal = 1.0, 2.0, 0.2, 10.0
    for i in range(nseg):
        for j in range(4):
            cp.coef[i][j] = float(coef[i, j])
    lk = rng.uniform(np.log(k_range[0]), np.log(k_range[1]), size=N)
    lh = rng.uniform(np.log(h_range[0]), np.log(h_range[1]), size=N)
    Ks = np.round(np.exp(lk)).astype(np.uint32)
    Hs = np.round(np.exp(lh)).astype(np.uint32)
    x0 = np.zeros((N, 5), np.float32)
    x0[:, 0] = rng.uniform(0.0, 20.0, size=N)
    for a in range(N):
        i = min(int(x0[a, 0] // dx), nseg - 1)
        sg = x0[a, 0] - i * dx
        x0[a, 1] = coef[i, 0] + sg * (coef[i, 1] + sg * (coef[i, 2] + sg * coef[i, 3])) \
            + rng.uniform(-1.0, 1.0)
        x0[a, 3] = rng.uniform(2.0, 6.0)
    covs = np.stack([_random_spd(rng, 0.05, 0.5) for _ in range(N)]).astype(np.float32)
    shared = np.diag([0.25, 0.25]).astype(np.float32)
    w = Workload("bicycle_uneven", "bicycle_lane", "bicycle_lane", 5, 2, int(Hs.max()),
                 int(Ks.max()), 1.0, shared, np.linalg.inv(shared).astype(np.float32),
                 np.array([-3.0, -0.5], np.float32), np.array([3.0, 0.5], np.float32), N, T,
                 x0, blob(mp), [blob(cp)] * N, covs.reshape(N, 4), cov_full=True, seed=seed)
    w.agent_K = Ks
    w.agent_H = Hs
    return w


def bicycle_executed_cost(states: np.ndarray, terminal: np.ndarray, cost_blob: bytes) -> np.ndarray:
    """Closed-loop lane-keeping cost of executed bicycle trajectories, per
    agent: the stage cost over x_1..x_T plus the terminal cost of x_T."""
    c = BicycleCostParams.from_buffer_copy(cost_blob)
    coef = np.array([[c.coef[i][j] for j in range(4)] for i in range(c.num_segments)])
    nxt = np.concatenate([states[1:], terminal[None]], axis=0).astype(np.float64)
    x = np.clip(nxt[..., 0], c.x0, c.x0 + c.knot_dx * c.num_segments)
    i = np.clip(np.floor((x - c.x0) / c.knot_dx).astype(int), 0, c.num_segments - 1)
    sg = x - (c.x0 + c.knot_dx * i)
    k = coef[i]
    yc = k[..., 0] + sg * (k[..., 1] + sg * (k[..., 2] + sg * k[..., 3]))
    slope = k[..., 1] + sg * (2.0 * k[..., 2] + sg * 3.0 * k[..., 3])
    st = (c.w_lat * (nxt[..., 1] - yc) ** 2 + c.w_head * (nxt[..., 2] - np.arctan(slope)) ** 2
          + c.w_speed * (nxt[..., 3] - c.v_ref) ** 2)
    return st.sum(axis=0) + c.w_terminal * st[-1]


def executed_cost(w: Workload, states, controls, terminal) -> np.ndarray:
    """Executed closed-loop cost per agent for the shipped benchmark models."""
    if w.plugin == "unicycle_obstacles":
        blobs = w.cost_params if len(w.cost_params) == states.shape[1] else \
            [w.cost_params[0]] * states.shape[1]
        return unicycle_executed_cost(states, controls, terminal, blobs)
    if w.plugin == "bicycle_lane":
        return bicycle_executed_cost(states, terminal, w.cost_params[0])
    if w.plugin == "quadrotor":
        return np.array([quadrotor_executed_cost(states[:, a], terminal[a], w.cost_params[a])
                         for a in range(states.shape[1])])
    return np.full(states.shape[1], np.nan)


def quadrotor_executed_cost(states: np.ndarray, terminal: np.ndarray, cost_blob: bytes) -> float:
    """Closed-loop cost of one executed quadrotor trajectory (states [T][12],
    terminal [12]): stage cost over x_1..x_T plus terminal cost of x_T."""
    c = QuadrotorCostParams.from_buffer_copy(cost_blob)
    nxt = np.concatenate([states[1:], terminal[None]], axis=0).astype(np.float64)
    p = nxt[:, 0:3]
    pos = c.w_pos * np.sum((p - np.array([c.wp_x, c.wp_y, c.wp_z])) ** 2, axis=1)
    n = min(int(c.num_obs), QUAD_MAX_OBS)
    ctr = np.stack([np.array(c.obs_cx[:n]), np.array(c.obs_cy[:n]), np.array(c.obs_cz[:n])], 1)
    d = np.sqrt(np.sum((p[:, None, :] - ctr[None]) ** 2, axis=2))
    pen = np.maximum(np.array(c.obs_r[:n])[None] - d, 0.0).sum(axis=1)
    st = (pos + c.w_vel * np.sum(nxt[:, 3:6] ** 2, 1) + c.w_att * np.sum(nxt[:, 6:8] ** 2, 1)
          + c.w_rate * np.sum(nxt[:, 9:12] ** 2, 1) + c.w_obs * pen)
    return float(st.sum() + c.w_terminal * pos[-1])


def quadrotor_batch(seed: int = 0, N: int = 32, K: int = 65536, H: int = 100, T: int = 100,
                    n_obs: int = 32) -> Workload:
    """Large rollout: N 12-state quadrotors (position, velocity, Euler
    angles, body rates; four rotor thrusts in [0, 2 * hover]), dt 0.01,
    H 100, K 65536, waypoint tracking and 32 spherical obstacles per agent."""
    rng = np.random.default_rng(seed)
    mp = QuadrotorModelParams(0.01, 1.0, 9.81, 0.25, 0.02, 0.01, 0.01, 0.02)
    hover = 1.0 * 9.81 / 4.0
    x0 = np.zeros((N, 12), np.float32)
    x0[:, 0:2] = rng.uniform(-4.0, 4.0, size=(N, 2))
    x0[:, 2] = 1.0
    cps = []
    for _ in range(N):
        c = QuadrotorCostParams()
        c.wp_x, c.wp_y = (float(v) for v in rng.uniform(-4.0, 4.0, size=2))
        c.wp_z = float(rng.uniform(1.0, 3.0))
        c.w_pos, c.w_vel, c.w_att, c.w_rate = 1.0, 0.1, 0.1, 0.01
        c.w_obs, c.w_terminal = 1.0e3, 10.0
        c.num_obs = n_obs
        for i in range(n_obs):
            c.obs_cx[i], c.obs_cy[i] = (float(v) for v in rng.uniform(-5.0, 5.0, size=2))
            c.obs_cz[i] = float(rng.uniform(0.0, 4.0))
            c.obs_r[i] = float(rng.uniform(0.2, 0.6))
        cps.append(blob(c))
    sigma = np.full(4, 1.0, np.float32)
    return Workload("quadrotor_batch", "quadrotor", "quadrotor", 12, 4, H, K, 1.0, sigma,
                    (1.0 / sigma ** 2).astype(np.float32), np.zeros(4, np.float32),
                    np.full(4, 2.0 * hover, np.float32), N, T, x0, blob(mp), cps, None,
                    seed=seed)
