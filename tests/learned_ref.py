"""Float64 CPU restatement of the learned-proposal network (TEST INFRASTRUCTURE ONLY).

Same network as pseudoctimaging_b200/csrc/pct_learned.h: conv 2->16 and three conv 16->16 (3x3x3,
valid, bias, ReLU) over the two 9x9x9 patches scaled by 1/512, then three linear heads 16->11;
loss = sum over the three axes of the cross-entropy against the per-axis targets. Used to check
the GPU's forward/backward kernels (gradients) and targets.
"""
import numpy as np
import torch
import torch.nn.functional as F

C, CIN, AX, HEADS = 16, 2, 11, 33
SIZES = [("W1", (C, CIN, 3, 3, 3)), ("B1", (C,)), ("W2", (C, C, 3, 3, 3)), ("B2", (C,)),
         ("W3", (C, C, 3, 3, 3)), ("B3", (C,)), ("W4", (C, C, 3, 3, 3)), ("B4", (C,)),
         ("H", (HEADS, C)), ("HB", (HEADS,))]
IN_SCALE = 1.0 / 512.0


def unflatten(p):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    assert o == len(p)
    return out


def patches(img, atlas, samples, subject_of):
    """samples: [n][3] (subject, atlas, voxel); returns [n][2][9][9][9] float64 scaled inputs."""
    out = np.empty((len(samples), 2, 9, 9, 9))
    for i, (s, a, vox) in enumerate(samples):
        im, at = img[s], atlas[s]
        nz, nx, ny = im.shape
        z, x, y = vox // (nx * ny), (vox % (nx * ny)) // ny, vox % ny
        sl = (slice(z - 4, z + 5), slice(x - 4, x + 5), slice(y - 4, y + 5))
        out[i, 0] = im[sl] * IN_SCALE
        out[i, 1] = at[a][sl] * IN_SCALE
    return out


def loss_and_grads(params, x, targets):
    """Mean loss and mean gradient (flat, float64) of the batch."""
    ps = {k: torch.tensor(v, dtype=torch.float64, requires_grad=True)
          for k, v in unflatten(np.asarray(params, np.float64)).items()}
    h = torch.tensor(x, dtype=torch.float64)
    for i in range(1, 5):
        h = F.relu(F.conv3d(h, ps[f"W{i}"], ps[f"B{i}"]))
    feat = h.reshape(h.shape[0], C)
    logits = feat @ ps["H"].T + ps["HB"]
    t = torch.tensor(targets, dtype=torch.float64)
    loss = 0
    for a in range(3):
        lp = F.log_softmax(logits[:, a * AX:(a + 1) * AX], dim=1)
        loss = loss - (t[:, a * AX:(a + 1) * AX] * lp).sum(dim=1)
    loss = loss.mean()
    loss.backward()
    g = np.concatenate([ps[name].grad.numpy().reshape(-1) for name, _ in SIZES])
    return float(loss.detach()), g


def top32_float64(img, atlas_vol, vox, k=32):
    """Exact float64 SSD of all 11^3 offsets for one voxel; returns SSDs in offset order."""
    nz, nx, ny = img.shape
    z, x, y = vox // (nx * ny), (vox % (nx * ny)) // ny, vox % ny
    a = img[z - 1:z + 2, x - 1:x + 2, y - 1:y + 2].astype(np.float64)
    ssd = np.empty(11 ** 3)
    o = 0
    for dw in range(-5, 6):
        for du in range(-5, 6):
            for dv in range(-5, 6):
                b = atlas_vol[z + dw - 1:z + dw + 2, x + du - 1:x + du + 2,
                              y + dv - 1:y + dv + 2].astype(np.float64)
                ssd[o] = ((a - b) ** 2).sum()
                o += 1
    return ssd
