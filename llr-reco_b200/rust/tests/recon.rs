//! Device tests (need a CUDA device): `cargo test -- --ignored`.
use llr_b200::{cu_low_rank_approx_batch, llr_recon, signal_model, Cf32, Config, ModelDirection, Prox};

fn pseudo_random(n: usize, seed: u64) -> Vec<Cf32> {
    let mut s = seed;
    let mut next = || {
        s = s.wrapping_mul(6364136223846793005).wrapping_add(1442695040888963407);
        ((s >> 40) as f32 / (1u64 << 24) as f32) - 0.5
    };
    (0..n).map(|_| Cf32 { re: next(), im: next() }).collect()
}

#[test]
#[ignore]
fn rank_one_matrices_survive_the_rank_one_approximation() {
    let (m, n, batch) = (64usize, 9usize, 4usize);
    let u = pseudo_random(m * batch, 1);
    let v = pseudo_random(n * batch, 2);
    let mut a = vec![Cf32::default(); m * n * batch];
    for b in 0..batch {
        for j in 0..n {
            for i in 0..m {
                let (x, y) = (u[b * m + i], v[b * n + j]);
                a[b * m * n + j * m + i] = Cf32 { re: x.re * y.re - x.im * y.im, im: x.re * y.im + x.im * y.re };
            }
        }
    }
    let orig = a.clone();
    cu_low_rank_approx_batch(m, n, 1, batch, &mut a).unwrap();
    let err: f32 = a.iter().zip(&orig).map(|(p, q)| (p.re - q.re).powi(2) + (p.im - q.im).powi(2)).sum();
    let nrm: f32 = orig.iter().map(|q| q.re * q.re + q.im * q.im).sum();
    assert!(err.sqrt() <= 1e-5 * nrm.sqrt());
}

#[test]
#[ignore]
fn recon_lowers_the_data_consistency_residual() {
    let (nx, ny, nz, nq) = (16usize, 16usize, 16usize, 5usize);
    let vol = nx * ny * nz;
    let base = pseudo_random(vol, 3);
    let mut k: Vec<Cf32> = (0..vol * nq)
        .map(|e| { let s = 1.0 - 0.1 * (e / vol) as f32; Cf32 { re: s * base[e % vol].re, im: s * base[e % vol].im } })
        .collect();
    let zero = vec![[0f32; 3]; nq];
    signal_model(&mut k, &[nx, ny, nz], nq, &zero, &zero, ModelDirection::Forward).unwrap();
    for (e, v) in k.iter_mut().enumerate() {
        let (iy, iz) = ((e / nx) % ny, (e / (nx * ny)) % nz);
        if (iy + 2 * iz + e / vol) % 3 == 0 {
            *v = Cf32::default();   // a third of the ky-kz lines not sampled
        }
    }
    let cfg = Config::new([nx, ny, nz], nq, [4, 4, 4], Prox::SoftThreshold(0.0));
    let mut img = vec![Cf32::default(); vol * nq];
    let h = llr_recon(&cfg, &k, None, 10, 0.02, &mut img).unwrap();
    assert!(h.iter().all(|v| v.is_finite()));
    assert!(h[9] < h[0]);
}
