"""The learned warm start of steady obstacle-channel solves.

A 3D convolutional U-Net in BF16 (channels-last volumes; every 3x3x3 convolution, forward and both gradients, on the
tensor cores through include/lbm_b200_warmstart.h) is trained on steady states that the plain solver computes, and
predicts the steady velocity and density of a channel from its solid mask.  A solve then starts from the equilibrium
of the prediction (lbm_set_fluid_equilibrium) instead of rest, and the plain solver judges convergence to the same
steady residual (lbm_steady_solve), so a poor prediction costs time but never accuracy.

The obstacle channel: a duct with bounce-back walls on the planes y = 0, ny - 1 and z = 0, nz - 1, a Velocity inlet
u = (u_in, 0, 0) on x = 0 and a Density outlet rho = 1 on x = nx - 1, tau 0.6, no momentum removal, and 5-20 solid
spheres of radius U[4, 10] with centres uniform in the interior (x in [12, nx - 12], the sphere inside the duct's
cross-section), all in lattice units.  Network input channels: the solid mask, the inlet velocity / 0.02, and the
coordinates x/nx, y/ny, z/nz (zero padding to 8); outputs: u/u_in and (rho - 1)/rho_scale.

The network that bench.py's time-to-steady measurement loads is trained by openmm-lbm_b200/warmstart_net/train.py,
which writes it beside itself (weights.pt).
"""
import argparse
import ctypes
import json
import threading
import time

import numpy as np
import torch

from .abi import MEMORY_DEVICE, check, load_library  # noqa: F401
from .force import LBMForce
from .kernel import B200Kernel

_SIGNATURES = {
    'lbm_conv3d_forward': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    'lbm_conv3d_weight_grad': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_void_p]),
    'lbm_conv3d_status': (ctypes.c_int, [ctypes.c_void_p]),
    'lbm_conv3d_set_wait_limit': (ctypes.c_int, [ctypes.c_longlong]),
}

INLET_SCALE = 0.02
IN_CHANNELS = 8


def _lib():
    lib = load_library()
    if not getattr(lib, '_warmstart_bound', False):
        for name, (restype, argtypes) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        lib._warmstart_bound = True
    return lib


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _volume(t):
    """(N, C, D, H, W) tensor with channels-last storage, as the kernels address it ([n][d][h][w][c])."""
    return t.contiguous(memory_format=torch.channels_last_3d)


def conv3d_forward(x, w, bias=None, relu=False):
    """y = conv3d(x, w) + bias (then ReLU): x (N, cin, D, H, W) BF16 channels-last, w (cout, 27, cin) BF16."""
    lib = _lib()
    x = _volume(x)
    n, cin, d, h, wd = x.shape
    cout = w.shape[0]
    w = w.contiguous()
    y = torch.empty((n, cout, d, h, wd), device=x.device, dtype=torch.bfloat16, memory_format=torch.channels_last_3d)
    b = bias.contiguous().float() if bias is not None else None
    check(lib.lbm_conv3d_forward(x.data_ptr(), w.data_ptr(), b.data_ptr() if b is not None else None, y.data_ptr(),
                                 n, d, h, wd, cin, cout, int(relu), _stream()), lib)
    return y


def conv3d_weight_grad(x, dy):
    """dW (cout, 27, cin) FP32 of y = conv3d(x, W) for the output gradient dy (BF16 channels-last)."""
    lib = _lib()
    x = _volume(x)
    dy = _volume(dy)
    n, cin, d, h, wd = x.shape
    cout = dy.shape[1]
    dw = torch.zeros((cout, 27, cin), device=x.device, dtype=torch.float32)
    check(lib.lbm_conv3d_weight_grad(x.data_ptr(), dy.data_ptr(), dw.data_ptr(), n, d, h, wd, cin, cout, _stream()),
          lib)
    return dw


def conv3d_input_grad(dy, w):
    """dX of y = conv3d(x, w): the forward convolution of dy with the flipped, transposed weights."""
    wt = w.flip(1).permute(2, 1, 0).contiguous()
    return conv3d_forward(dy, wt)


def conv_status():
    lib = _lib()
    check(lib.lbm_conv3d_status(_stream()), lib)


class Conv3dFunction(torch.autograd.Function):
    """BF16 3x3x3 convolution with FP32 master weights; the ReLU (when set) is fused into the forward kernel and its
    mask taken from the output in the backward pass."""

    @staticmethod
    def forward(ctx, x, weight, bias, relu):
        w16 = weight.to(torch.bfloat16)
        y = conv3d_forward(x, w16, bias, relu)
        ctx.save_for_backward(x, w16, y if relu else None)
        ctx.relu = relu
        return y

    @staticmethod
    def backward(ctx, dy):
        x, w16, y = ctx.saved_tensors
        dy = _volume(dy.to(torch.bfloat16))
        if ctx.relu:
            dy = _volume(dy*(y > 0).to(dy.dtype))
        dx = conv3d_input_grad(dy, w16) if ctx.needs_input_grad[0] else None
        dw = conv3d_weight_grad(x, dy)
        db = dy.float().sum(dim=(0, 2, 3, 4))
        return dx, dw, db, None


class WarmStartNet(torch.nn.Module):
    """U-Net: per level two convolutions with ReLU (widths 16, 32, 64, 160), 2x average pooling down, nearest 2x
    upsampling and concatenation with the skip up, a linear 3x3x3 head to 4 channels (padded to 16)."""

    def __init__(self, widths=(16, 32, 64, 160), in_channels=IN_CHANNELS, out_channels=4, seed=0):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.widths, self.out_channels = tuple(widths), out_channels
        self.weights, self.biases = torch.nn.ParameterList(), torch.nn.ParameterList()
        specs = []
        c = in_channels
        for w in widths:
            specs += [(c, w), (w, w)]
            c = w
        for level in range(len(widths) - 2, -1, -1):
            specs += [(widths[level + 1] + widths[level], widths[level]), (widths[level], widths[level])]
        specs.append((widths[0], 16))
        for cin, cout in specs:
            std = (2.0/(27*cin))**0.5
            self.weights.append(torch.nn.Parameter(torch.randn(cout, 27, cin, generator=g)*std))
            self.biases.append(torch.nn.Parameter(torch.zeros(cout)))
        with torch.no_grad():
            self.weights[-1].mul_(0.1)
        self.register_buffer('rho_scale', torch.tensor(1e-3))
        # Standardisation of the 4 outputs (u/u_in, (rho - 1)/rho_scale) over the fluid nodes of the training set.
        self.register_buffer('out_mean', torch.zeros(out_channels))
        self.register_buffer('out_std', torch.ones(out_channels))

    def parameter_count(self):
        return sum(p.numel() for p in self.weights) + sum(p.numel() for p in self.biases)

    def _conv(self, i, h, relu=True):
        return Conv3dFunction.apply(h, self.weights[i], self.biases[i], relu)

    def forward(self, x):
        levels = len(self.widths)
        skips, h, i = [], x, 0
        for level in range(levels):
            h = self._conv(i + 1, self._conv(i, h))
            i += 2
            if level < levels - 1:
                skips.append(h)
                h = _volume(torch.nn.functional.avg_pool3d(h, 2))
        for level in range(levels - 2, -1, -1):
            h = torch.nn.functional.interpolate(h, scale_factor=2, mode='nearest')
            h = _volume(torch.cat([h, skips[level]], dim=1))
            h = self._conv(i + 1, self._conv(i, h))
            i += 2
        return self._conv(i, h, relu=False)[:, :self.out_channels]


# ------------------------------------------------------------------------------------------------------------------
# Obstacle channels and their steady solves.
# ------------------------------------------------------------------------------------------------------------------

def obstacle_mask(seed, shape=(128, 64, 64), count=(5, 20), radius=(4.0, 10.0)):
    """Solid mask [z][y][x] of the duct walls and the seeded spheres."""
    nx, ny, nz = shape
    rng = np.random.Generator(np.random.PCG64(seed))
    spheres = int(rng.integers(count[0], count[1] + 1))
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing='ij')
    solid = (y == 0) | (y == ny - 1) | (z == 0) | (z == nz - 1)
    margin = min(12, nx//4)
    for _ in range(spheres):
        r = min(rng.uniform(*radius), (min(ny, nz) - 3)/2.0)
        c = (rng.uniform(margin, nx - margin), rng.uniform(r + 1, ny - 2 - r), rng.uniform(r + 1, nz - 2 - r))
        solid |= (x - c[0])**2 + (y - c[1])**2 + (z - c[2])**2 <= r*r
    return solid


def channel_lattice(shape=(128, 64, 64), inlet=0.02, tau=0.6):
    nx, ny, nz = shape
    force = LBMForce()
    force.setGridSize(nx, ny, nz)
    force.setFluidDensity(1.0)
    force.setKinematicViscosity((tau - 0.5)/3.0)
    force.setFluidMomentumRemovalFrequency(0)
    force.setFaceBoundary(LBMForce.XMin, LBMForce.Velocity)
    force.setFaceVelocity(LBMForce.XMin, (inlet, 0.0, 0.0))
    force.setFaceBoundary(LBMForce.XMax, LBMForce.Density)
    force.setFaceDensity(LBMForce.XMax, 1.0)
    return force.latticeParameters(np.array(shape, dtype=float), 1.0, np.ones(1))


def channel_kernel(solid, shape=(128, 64, 64), precision='single', inlet=0.02):
    return B200Kernel(channel_lattice(shape, inlet), [], np.nonzero(solid.ravel())[0], precision)


def network_input(masks, inlet=0.02):
    """(N, 8, nz, ny, nx) BF16 channels-last input of a batch of solid masks ([z][y][x] bool tensors on the device)."""
    n = len(masks)
    nz, ny, nx = masks[0].shape
    dev = masks[0].device
    x = torch.zeros((n, IN_CHANNELS, nz, ny, nx), device=dev, dtype=torch.float32)
    zz = torch.linspace(0, 1, nz, device=dev).view(nz, 1, 1)
    yy = torch.linspace(0, 1, ny, device=dev).view(1, ny, 1)
    xx = torch.linspace(0, 1, nx, device=dev).view(1, 1, nx)
    for i, m in enumerate(masks):
        x[i, 0] = m.float()
        x[i, 1] = inlet/INLET_SCALE
        x[i, 2] = xx.expand(nz, ny, nx)
        x[i, 3] = yy.expand(nz, ny, nx)
        x[i, 4] = zz.expand(nz, ny, nx)
    return _volume(x.to(torch.bfloat16))


def steady_target(kernel, solid, inlet, rho_scale):
    """(4, nz, ny, nx) FP32 target (u/u_in, (rho - 1)/rho_scale) of the kernel's fields; zero at solid nodes."""
    density, velocity = kernel.get_fluid_fields()
    shape = solid.shape
    fluid = ~solid
    t = np.zeros((4,) + shape, dtype=np.float32)
    for a in range(3):
        t[a] = np.where(fluid, velocity[:, a].reshape(shape)/inlet, 0.0)
    t[3] = np.where(fluid, (density.reshape(shape) - 1.0)/rho_scale, 0.0)
    return t


def solve_cases(seeds, shape, inlet, rho_scale, threads=4, tolerance=1e-6, max_steps=300000, radius=(4.0, 10.0)):
    """Cold steady solves of the cases, `threads` at a time (each kernel on its own stream): per seed the solid mask,
    the FP16 target, the steps and residual of the solve and its wall time (comparable between cases only with
    threads = 1)."""
    results = {}
    lock = threading.Lock()
    pending = list(seeds)

    def worker():
        while True:
            with lock:
                if not pending:
                    return
                seed = pending.pop(0)
            solid = obstacle_mask(seed, shape, radius=radius)
            kernel = channel_kernel(solid, shape, inlet=inlet)
            t0 = time.perf_counter()
            steps, r = kernel.solve_steady(0, 100, tolerance, max_steps)
            seconds = time.perf_counter() - t0
            target = steady_target(kernel, solid, inlet, rho_scale).astype(np.float16)
            kernel.close()
            with lock:
                results[seed] = (solid, target, steps, r, seconds)

    pool = [threading.Thread(target=worker) for _ in range(threads)]
    for t in pool:
        t.start()
    for t in pool:
        t.join()
    return results


def predict_fields(net, solid, inlet):
    """Predicted density [N] and velocity [N][3] (float64 CUDA tensors, node order x fastest) of one case."""
    with torch.no_grad():
        mask = torch.as_tensor(solid, device='cuda')
        out = net(network_input([mask], inlet))[0].float()*net.out_std.view(-1, 1, 1, 1) + net.out_mean.view(-1, 1, 1, 1)
        fluid = (~mask).float()
        u = out[:3]*inlet*fluid
        rho = 1.0 + out[3]*net.rho_scale*fluid
        velocity = u.permute(1, 2, 3, 0).contiguous().double().view(-1, 3)
        density = rho.contiguous().double().view(-1)
    return density, velocity


def train(net, cases, epochs, batch=2, lr=2e-3, log=None):
    """Adam on the mean squared error over the fluid nodes of the normalised fields."""
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    seeds = sorted(cases)
    masks = {s: torch.as_tensor(cases[s][0], device='cuda') for s in seeds}
    targets = {s: torch.as_tensor(cases[s][1], device='cuda').to(torch.bfloat16) for s in seeds}
    rng = np.random.Generator(np.random.PCG64(7))
    with torch.no_grad():
        count, total, total2 = 0.0, torch.zeros(4, device='cuda'), torch.zeros(4, device='cuda')
        for s in seeds:
            f = (~masks[s]).float()
            t = targets[s].float()
            count += float(f.sum())
            total += (t*f).sum(dim=(1, 2, 3))
            total2 += (t*t*f).sum(dim=(1, 2, 3))
        mean = total/count
        net.out_mean.copy_(mean)
        net.out_std.copy_(torch.sqrt(torch.clamp(total2/count - mean*mean, min=1e-12)))
    steps = epochs*max(1, len(seeds)//batch)
    sched = torch.optim.lr_scheduler.OneCycleLR(opt, max_lr=lr, total_steps=steps, pct_start=0.1)
    history = []
    for epoch in range(epochs):
        order = rng.permutation(seeds)
        total = 0.0
        for i in range(0, len(order) - batch + 1, batch):
            chunk = order[i:i + batch]
            x = network_input([masks[s] for s in chunk])
            y = (torch.stack([targets[s] for s in chunk]).float() - net.out_mean.view(1, -1, 1, 1, 1)) \
                / net.out_std.view(1, -1, 1, 1, 1)
            fluid = torch.stack([~masks[s] for s in chunk]).unsqueeze(1).float()
            pred = net(x).float()
            loss = (((pred - y)**2)*fluid).sum()/(fluid.sum()*4)
            opt.zero_grad()
            loss.backward()
            opt.step()
            sched.step()
            total += float(loss.detach())
        history.append(total/max(1, len(order)//batch))
        if log:
            log('epoch %d loss %.4e' % (epoch, history[-1]))
    conv_status()
    return history


def evaluate(net, cases, shape, inlet, tolerance=1e-6, max_steps=300000):
    """Warm-started solves of the held-out cases against their cold solves: wall time, steps, final-field error."""
    rows = []
    for seed in sorted(cases):
        solid, target, cold_steps, cold_r, cold_seconds = cases[seed]
        kernel = channel_kernel(solid, shape, inlet=inlet)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        density, velocity = predict_fields(net, solid, inlet)
        torch.cuda.synchronize()
        t_predict = time.perf_counter() - t0
        kernel.set_fluid_equilibrium(density, velocity)
        steps, r = kernel.solve_steady(0, 100, tolerance, max_steps)
        warm_seconds = time.perf_counter() - t0
        warm = steady_target(kernel, solid, inlet, float(net.rho_scale))
        kernel.close()
        target = target.astype(np.float32)
        fluid = ~solid
        err = np.sqrt(sum(((warm[a] - target[a])[fluid]**2).sum() for a in range(3))
                      / sum((target[a][fluid]**2).sum() for a in range(3)))
        rows.append({'seed': int(seed), 'cold_steps': int(cold_steps), 'cold_seconds': cold_seconds,
                     'warm_steps': int(steps), 'warm_seconds': warm_seconds, 'predict_seconds': t_predict,
                     'speedup': cold_seconds/warm_seconds, 'final_velocity_error': float(err),
                     'cold_residual': float(cold_r), 'warm_residual': float(r)})
    return rows


def conv_benchmark(shape=(128, 64, 64), widths=(16, 32, 64, 160), batch=2, repeats=5):
    """Device time (CUDA events) of the forward and weight-gradient convolutions of every layer shape of the U-Net at
    `shape` and `batch`: per layer the FLOPs (2 x voxels x 27 cin x cout per pass) and the TFLOP/s reached."""
    nx, ny, nz = shape
    layers, c = [], IN_CHANNELS
    for level, w in enumerate(widths):
        s = 2**level
        layers += [((nz//s, ny//s, nx//s), c, w), ((nz//s, ny//s, nx//s), w, w)]
        c = w
    for level in range(len(widths) - 2, -1, -1):
        s = 2**level
        layers += [((nz//s, ny//s, nx//s), widths[level + 1] + widths[level], widths[level]),
                   ((nz//s, ny//s, nx//s), widths[level], widths[level])]
    layers.append(((nz, ny, nx), widths[0], 16))
    rows = []
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for (d, h, w), cin, cout in layers:
        x = _volume(torch.randn((batch, cin, d, h, w), device='cuda').to(torch.bfloat16))
        wt = (torch.randn((cout, 27, cin), device='cuda')*0.1).to(torch.bfloat16)
        dy = _volume(torch.randn((batch, cout, d, h, w), device='cuda').to(torch.bfloat16))
        flops = 2.0*batch*d*h*w*27*cin*cout
        times = {}
        for name, fn in (('forward', lambda: conv3d_forward(x, wt)), ('weight_grad', lambda: conv3d_weight_grad(x, dy))):
            fn()
            torch.cuda.synchronize()
            start.record()
            for _ in range(repeats):
                fn()
            stop.record()
            torch.cuda.synchronize()
            times[name] = start.elapsed_time(stop)/repeats
        rows.append({'volume': [d, h, w], 'cin': cin, 'cout': cout, 'gflop': flops/1e9,
                     'forward_ms': times['forward'], 'forward_tflops': flops/(times['forward']*1e-3)/1e12,
                     'weight_grad_ms': times['weight_grad'],
                     'weight_grad_tflops': flops/(times['weight_grad']*1e-3)/1e12})
    conv_status()
    return rows


def save_network(net, path):
    """The network's weights (BF16, the precision the convolutions use), biases, output standardisation and widths."""
    torch.save({'widths': list(net.widths),
                'weights': [w.detach().to(torch.bfloat16).cpu() for w in net.weights],
                'biases': [b.detach().float().cpu() for b in net.biases],
                'rho_scale': float(net.rho_scale), 'out_mean': net.out_mean.cpu(), 'out_std': net.out_std.cpu()}, path)


def load_network(path):
    """A WarmStartNet on the GPU with the weights that save_network wrote."""
    data = torch.load(path, map_location='cpu')
    net = WarmStartNet(widths=tuple(data['widths']))
    with torch.no_grad():
        for p, w in zip(net.weights, data['weights']):
            p.copy_(w.float())
        for p, b in zip(net.biases, data['biases']):
            p.copy_(b)
        net.rho_scale.fill_(data['rho_scale'])
        net.out_mean.copy_(data['out_mean'])
        net.out_std.copy_(data['out_std'])
    return net.cuda()


def time_to_steady(net, seeds, shape=(128, 64, 64), inlet=0.02, tolerance=1e-6, radius=(4.0, 10.0)):
    """Held-out channels solved to the steady residual `tolerance` from rest and from the network's prediction, one
    after the other: per case the wall time (the prediction included) and the steps of each, and the warm solve's
    final velocity error against the cold one."""
    cases = solve_cases(seeds, shape, inlet, float(net.rho_scale), threads=1, tolerance=tolerance, radius=radius)
    return evaluate(net, cases, shape, inlet, tolerance=tolerance)


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument('--train', type=int, default=2000)
    p.add_argument('--test', type=int, default=200)
    p.add_argument('--epochs', type=int, default=8)
    p.add_argument('--batch', type=int, default=2)
    p.add_argument('--shape', default='128x64x64')
    p.add_argument('--widths', default='16,32,64,160')
    p.add_argument('--threads', type=int, default=4, help='concurrent solves of the training data')
    p.add_argument('--radius', default='4,10', help='sphere radii range')
    p.add_argument('--out', default='warmstart_report.json')
    p.add_argument('--save', default='', help='write the trained network (save_network) to this path')
    p.add_argument('--no-conv-benchmark', action='store_true')
    args = p.parse_args(argv)
    shape = tuple(int(a) for a in args.shape.split('x'))
    inlet = 0.02
    log = lambda s: print(s, flush=True)  # noqa: E731
    t0 = time.perf_counter()
    train_seeds = list(range(1, args.train + 1))
    test_seeds = list(range(100001, 100001 + args.test))
    rho_scale = 1e-3
    radius = tuple(float(r) for r in args.radius.split(','))
    train_cases = solve_cases(train_seeds, shape, inlet, rho_scale, args.threads, radius=radius)
    # The held-out cold solves run one at a time: their wall times are the baseline of the warm starts.
    test_cases = solve_cases(test_seeds, shape, inlet, rho_scale, 1, radius=radius)
    t_data = time.perf_counter() - t0
    log('data: %d + %d steady solves in %.1f s' % (len(train_cases), len(test_cases), t_data))
    net = WarmStartNet(widths=tuple(int(w) for w in args.widths.split(','))).cuda()
    t1 = time.perf_counter()
    history = train(net, train_cases, args.epochs, args.batch, log=log)
    t_train = time.perf_counter() - t1
    if args.save:
        save_network(net, args.save)
    rows = evaluate(net, test_cases, shape, inlet)
    speedups = np.array([r['speedup'] for r in rows])
    errors = np.array([r['final_velocity_error'] for r in rows])
    report = {'shape': shape, 'train': len(train_cases), 'test': len(test_cases), 'epochs': args.epochs,
              'parameters': net.parameter_count(), 'data_seconds': t_data, 'train_seconds': t_train,
              'loss_history': history,
              'speedup_mean': float(speedups.mean()), 'speedup_median': float(np.median(speedups)),
              'speedup_min': float(speedups.min()),
              'time_ratio_total': float(sum(r['cold_seconds'] for r in rows)/sum(r['warm_seconds'] for r in rows)),
              'steps_ratio_total': float(sum(r['cold_steps'] for r in rows)/max(1, sum(r['warm_steps'] for r in rows))),
              'final_velocity_error_max': float(errors.max()), 'final_velocity_error_mean': float(errors.mean()),
              'cases': rows}
    if not args.no_conv_benchmark:
        report['conv_benchmark'] = conv_benchmark(shape, tuple(int(w) for w in args.widths.split(',')), args.batch)
    with open(args.out, 'w') as f:
        json.dump(report, f)
    log(json.dumps({k: v for k, v in report.items() if k not in ('cases', 'loss_history', 'conv_benchmark')}))
    return report


if __name__ == '__main__':
    main()
