//! Exports reference values for the parity oracle of nightstream_b200 (see
//! Cargo.toml).  Every value is produced by the reference's own code path:
//! `neo_ccs::crypto::poseidon2_goldilocks::permutation()` (the transcript
//! permutation), `Poseidon2Goldilocks::<16>::new_from_rng_128` seeded as
//! `digest_ccs_matrices` seeds it, `neo_ajtai::setup_par`, and
//! `Poseidon2Transcript`.  Output: one JSON object, every field element as a
//! decimal string of its canonical u64.
use neo_ccs::crypto::poseidon2_goldilocks as p2;
use neo_transcript::{Poseidon2Transcript, Transcript};
use p3_field::{PrimeCharacteristicRing, PrimeField64};
use p3_goldilocks::{Goldilocks, Poseidon2Goldilocks};
use p3_symmetric::Permutation;
use rand_chacha::rand_core::{RngCore, SeedableRng};
use rand_chacha::ChaCha8Rng;

const CCS_DIGEST_SEED: u64 = 0x434353445F4D4154;
const PP_SEED: [u8; 32] = [7u8; 32];
const PP_KAPPA: usize = 16;
const PP_M: usize = 64;

fn list(xs: impl IntoIterator<Item = u64>) -> String {
    let v: Vec<String> = xs.into_iter().map(|x| format!("\"{x}\"")).collect();
    format!("[{}]", v.join(", "))
}

fn canon(xs: &[Goldilocks]) -> String {
    list(xs.iter().map(|x| x.as_canonical_u64()))
}

fn main() {
    // width-8 transcript permutation applied to [0, 1, ..., 7]
    let s8: [Goldilocks; 8] = core::array::from_fn(|i| Goldilocks::from_u64(i as u64));
    let p8 = p2::permutation().permute(s8);
    // width-16 digest permutation applied to [0, 1, ..., 15]
    let mut rng16 = ChaCha8Rng::seed_from_u64(CCS_DIGEST_SEED);
    let perm16 = Poseidon2Goldilocks::<16>::new_from_rng_128(&mut rng16);
    let s16: [Goldilocks; 16] = core::array::from_fn(|i| Goldilocks::from_u64(i as u64));
    let p16 = perm16.permute(s16);
    // the ChaCha8 streams the two permutations' constants are drawn from
    let mut c8 = ChaCha8Rng::from_seed(p2::SEED);
    let stream8: Vec<u64> = (0..64).map(|_| c8.next_u64()).collect();
    let mut c16 = ChaCha8Rng::seed_from_u64(CCS_DIGEST_SEED);
    let stream16: Vec<u64> = (0..64).map(|_| c16.next_u64()).collect();
    // setup_par PP: row 0, columns 0 and m - 1 (54 coefficients each), and row kappa - 1, column 0
    let mut pp_rng = ChaCha8Rng::from_seed(PP_SEED);
    let pp = neo_ajtai::setup_par(&mut pp_rng, neo_math::D, PP_KAPPA, PP_M).expect("setup_par");
    let col = |i: usize, j: usize| canon(&neo_math::cf(pp.m_rows[i][j]));
    // transcript: new(b"neo/bench"), then one challenge_field(b"golden/chal")
    let mut tr = Poseidon2Transcript::new(b"neo/bench");
    let st0 = tr.state();
    let ch = tr.challenge_field(b"golden/chal");
    let st1 = tr.state();

    println!("{{");
    println!("  \"poseidon2_w8_seed\": {},", list(p2::SEED.iter().map(|&b| b as u64)));
    println!("  \"poseidon2_w8_permute_0_to_7\": {},", canon(&p8));
    println!("  \"poseidon2_w16_permute_0_to_15\": {},", canon(&p16));
    println!("  \"chacha8_from_seed_w8_seed_first_64\": {},", list(stream8));
    println!("  \"chacha8_seed_from_u64_ccs_digest_first_64\": {},", list(stream16));
    println!("  \"pp_seed\": {},", list(PP_SEED.iter().map(|&b| b as u64)));
    println!("  \"pp_kappa\": {PP_KAPPA},");
    println!("  \"pp_m\": {PP_M},");
    println!("  \"pp_setup_par_row0_col0\": {},", col(0, 0));
    println!("  \"pp_setup_par_row0_col_last\": {},", col(0, PP_M - 1));
    println!("  \"pp_setup_par_row_last_col0\": {},", col(PP_KAPPA - 1, 0));
    println!("  \"transcript_app_label\": \"neo/bench\",");
    println!("  \"transcript_state_after_new\": {},", canon(&st0));
    println!("  \"transcript_challenge_label\": \"golden/chal\",");
    println!("  \"transcript_challenge\": \"{}\",", ch.as_canonical_u64());
    println!("  \"transcript_state_after_challenge\": {}", canon(&st1));
    println!("}}");
}
