"""MLP warm start for quasi-static FIRE load increments.

Training pairs come from plain-FIRE increments of an engine: the per-particle features
before an increment (rf_engine_warm_features) and the relaxed displacement and rotation
after it (rf_engine_warm_targets). The MLP (rf_mlp_*, tensor-core BF16 forward and
backward) learns the correction to the last increment's motion; a prediction is applied
with rf_engine_load_increment_pred, and FIRE then relaxes to the same residual tolerance
as plain FIRE, which remains the fallback.
"""
import numpy as np

from . import MLP, check, lib, ptr


class WarmStart:
    def __init__(self, n_particles, strain_inc, seed=0xB2000000, residual=True):
        import torch
        self.torch = torch
        self.N = int(n_particles)
        self.rows = (self.N + 127) // 128 * 128
        self.strain_inc = float(strain_inc)
        self.mlp = MLP(seed)
        self.mlp.set_residual(residual)
        self.feat = torch.zeros(self.rows, 64, dtype=torch.bfloat16, device="cuda")
        self.tgt = torch.zeros(self.N, 6, device="cuda")
        self.Y = torch.zeros(self.rows, 16, device="cuda")
        self.X, self.T = [], []

    def features(self, engine):
        """Features of `engine` for its next increment (kept for collect())."""
        engine.warm_features(self.strain_inc, self.feat)
        self.torch.cuda.synchronize()
        return self.feat

    def collect(self, engine):
        """After a plain increment whose features were taken with features(): store the pair."""
        engine.warm_targets(self.strain_inc, self.tgt)
        self.torch.cuda.synchronize()
        self.X.append(self.feat[: self.N].clone())
        self.T.append(self.tgt.clone())

    def pairs(self):
        return sum(x.shape[0] for x in self.X)

    def train(self, steps=400, lr=2e-3, lr_final=5e-4):
        X = self.torch.cat(self.X)
        T = self.torch.cat(self.T)
        # the concatenations run on torch's stream, the training steps on the MLP's own
        self.torch.cuda.synchronize()
        rows = X.shape[0]
        losses = []
        for it in range(steps):
            a = lr if it < (2 * steps) // 3 else lr_final
            losses.append(self.mlp.train_step(X, T, rows, a))
        return losses

    def predict(self, engine, rotations=False):
        """The prediction for `engine`'s next increment: float32 [rows, 16] on the device.
        The engine and the MLP run on their own streams: each hand-over synchronises.
        rotations=False starts the particles' rotations from zero instead of the predicted
        ones: the converged rotations change much from one increment to the next, and
        with a displacement prediction that is not exact, zero rotations let FIRE
        converge in fewer iterations (measured on the 200k bench specimen: with the last
        increment's displacements, 915 iterations with zero rotations, 1604 with the exact
        rotations; 1759 plain)."""
        self.features(engine)
        self.torch.cuda.synchronize()
        self.mlp.forward(self.feat, self.N, self.Y)
        # the forward pass runs on the MLP's stream: finish it before torch's stream
        # touches Y (the engine reads Y on its own stream after this returns)
        self.torch.cuda.synchronize()
        if not rotations:
            self.Y[:, 3:6] = 0.0
        self.torch.cuda.synchronize()
        return self.Y

    def close(self):
        self.mlp.close()
