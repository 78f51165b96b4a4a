"""MLP warm start for quasi-static FIRE load increments.

A warm start predicts each particle's motion over the next load increment; the engine
applies it (rf_engine_load_increment_pred) and FIRE then relaxes to the same residual
tolerance as plain FIRE, so a prediction only changes how many iterations that takes.

The base prediction is the last increment's motion, taken exactly (float) from the
engine (rf_engine_warm_targets before the increment), with a particle's translation
capped at base_cap platen advances (a particle that rearranged in the last increment
is not thrown as far again). The MLP (rf_mlp_*, tensor-core
BF16 forward and backward) learns the correction to it: training pairs are the
per-particle features before a plain increment (rf_engine_warm_features) and the
increment's relaxed motion less the last increment's. A correction is clamped
component-wise to a few RMS of the training corrections, so an outlier cannot throw a
particle into its neighbours.

A gate keeps the MLP honest: after every warm-started increment the MLP's prediction
and the last increment's motion are both compared with the relaxed motion, and the next
increment uses the MLP only while its error is below `gate` times the base's. The
newest pairs can also be added to the training set (observe(..., learn=True)).
"""
import numpy as np

from . import MLP


class WarmStart:
    def __init__(self, n_particles, strain_inc, seed=0xB2000000, clamp=4.0, gate=0.8, base_cap=2.0):
        import torch
        self.torch = torch
        self.N = int(n_particles)
        self.rows = (self.N + 127) // 128 * 128
        self.strain_inc = float(strain_inc)
        self.clamp = float(clamp)
        self.gate = float(gate)
        self.base_cap = float(base_cap)
        self.mlp = MLP(seed)
        self.mlp.set_residual(False)
        self.feat = torch.zeros(self.rows, 64, dtype=torch.bfloat16, device="cuda")
        self.tgt = torch.zeros(self.N, 6, device="cuda")
        self.Y = torch.zeros(self.rows, 16, device="cuda")
        self.L = None            # the last increment's motion of the engine features() last saw
        self.corr = None         # the MLP's clamped correction of the last predict()
        self.X, self.T = [], []  # training features and corrections
        self.cmax = None         # per-component clamp of the corrections
        self.use_mlp = True      # the gate's decision for the next prediction
        self.log = []            # per observed increment: (MLP error / base error, MLP used)
        self.base_error = []     # per observed increment: |last motion - relaxed motion| / |relaxed motion|

    def _motion(self, engine):
        """The motion of `engine`'s last increment, [N, 6] float32 (units of the increment)."""
        engine.warm_targets(self.strain_inc, self.tgt)
        self.torch.cuda.synchronize()
        return self.tgt.clone()

    def features(self, engine):
        """Features of `engine` for its next increment and its last increment's motion
        (kept for collect() / predict()). Needs one increment done."""
        engine.warm_features(self.strain_inc, self.feat)
        self.torch.cuda.synchronize()
        self.L = self._motion(engine)
        return self.feat

    def collect(self, engine):
        """After a plain increment whose features were taken with features(): store the
        pair (features, relaxed motion - last motion)."""
        T = self._motion(engine)
        self.X.append(self.feat[: self.N].clone())
        self.T.append(T - self.L)

    def pairs(self):
        return sum(x.shape[0] for x in self.X)

    def train(self, steps=400, lr=2e-3, lr_final=5e-4):
        X = self.torch.cat(self.X)
        T = self.torch.cat(self.T)
        self.cmax = self.clamp * T.pow(2).mean(0).sqrt() + 1e-12
        # the concatenations run on torch's stream, the training steps on the MLP's own
        self.torch.cuda.synchronize()
        rows = X.shape[0]
        losses = []
        for it in range(steps):
            a = lr if it < (2 * steps) // 3 else lr_final
            losses.append(self.mlp.train_step(X, T, rows, a))
        return losses

    def predict(self, engine, use_mlp=None, rotations=False):
        """The prediction for `engine`'s next increment: float32 [rows, 16] on the device
        (columns 0-5: displacement and rotation in units of the increment). use_mlp: None
        follows the gate, False gives the last increment's motion alone. rotations=False
        starts the particles' rotations from zero: the relaxed rotations change much from
        one increment to the next (measured on a 200k-particle specimen: with the last
        increment's displacements, 915 iterations with zero rotations, 1604 with the exact
        rotations; 1759 plain). The engine and the MLP run on their own streams: each
        hand-over synchronises."""
        self.features(engine)
        if self.base_cap > 0:
            # a particle that rearranged in the last increment (moved further than base_cap
            # platen advances) is not thrown that far again: its base motion is scaled down
            n = self.L[:, :3].norm(dim=1, keepdim=True)
            self.L[:, :3] *= self.torch.clamp(self.base_cap / self.torch.clamp(n, min=1e-30), max=1.0)
        use = self.use_mlp if use_mlp is None else bool(use_mlp)
        if use_mlp is False:
            self.corr = None                  # the base alone: no forward pass
            self.Y[: self.N, :6] = self.L
        else:
            # (with the gate closed the correction is still formed: observe() scores it)
            self.mlp.forward(self.feat, self.N, self.Y)
            # the forward pass runs on the MLP's stream: finish it before torch's stream
            # touches Y (the engine reads Y on its own stream after this returns)
            self.torch.cuda.synchronize()
            corr = self.Y[: self.N, :6]
            if self.cmax is not None:
                corr = self.torch.maximum(self.torch.minimum(corr, self.cmax), -self.cmax)
            self.corr = corr.clone()
            self.Y[: self.N, :6] = self.L + (self.corr if use else 0.0)
        if not rotations:
            self.Y[:, 3:6] = 0.0
        self.torch.cuda.synchronize()
        self.last_used = use
        return self.Y

    def observe(self, engine, learn=False, steps=20, lr=5e-4):
        """After the increment predict() prepared: compare the MLP's and the base's
        translation errors against the relaxed motion and set the gate for the next
        prediction; with learn=True the pair joins the training set and the MLP takes a
        few steps on the newest pairs."""
        if self.corr is None:
            raise ValueError("observe() follows a predict() that formed the MLP's correction")
        T = self._motion(engine)
        e_mlp = float((self.L[:, :3] + self.corr[:, :3] - T[:, :3]).pow(2).sum())
        e_base = float((self.L[:, :3] - T[:, :3]).pow(2).sum())
        ratio = np.sqrt(e_mlp / e_base) if e_base > 0 else 1.0
        self.log.append((ratio, self.last_used))
        t2 = float(T[:, :3].pow(2).sum())
        self.base_error.append(np.sqrt(e_base / t2) if t2 > 0 else 0.0)
        self.use_mlp = ratio < self.gate
        if learn:
            self.X.append(self.feat[: self.N].clone())
            self.T.append(T - self.L)
            X = self.torch.cat(self.X[-2:])
            Tc = self.torch.cat(self.T[-2:])
            self.torch.cuda.synchronize()
            for _ in range(steps):
                self.mlp.train_step(X, Tc, X.shape[0], lr)
        return ratio

    def close(self):
        self.mlp.close()
