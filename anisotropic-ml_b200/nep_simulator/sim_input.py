"""Command line of the simulator (reference: ``nep_simulator/sim_input.py``).

Same mandatory flags and output location (``./out/<out>.gsd``) as the
reference, for example
  python sim_input.py --init ./init/th_init_N200.gsd --out th05 --ts 20000 --dump 1000 \
      --kT 0.5 --dt 0.005 --model_path ./models/model_th_C100.pth --gpu_id 0 \
      --hypers 10 10 10 4.5 --shape th_v1
Optional flags (not in the reference): --method {fd,fd_split,adjoint},
--activation {relu,tanh,silu}, --nn_width, --nn_hidden, --nve.
"""
import argparse
import os

from NVT import NVT


def main(argv=None):
    parser = argparse.ArgumentParser(description="Runs NN-assisted MD")
    non_opt = parser.add_argument_group("mandatory arguments")
    non_opt.add_argument("--init", metavar="<dat>", type=str, dest="init_gsd", required=True, help=".gsd files ")
    non_opt.add_argument("--out", metavar="<dat>", type=str, dest="output", required=True, help=".gsd files ")
    non_opt.add_argument("--ts", metavar="<int>", type=int, dest="timesteps", required=True, help="length of sim ")
    non_opt.add_argument("--dump", metavar="<int>", type=int, dest="dump_period", required=True,
                         help="dump frequency ")
    non_opt.add_argument("--kT", metavar="<float>", type=float, dest="kT", required=True, help="temperature ")
    non_opt.add_argument("--dt", metavar="<float>", type=float, dest="dt", required=True, help="dt ")
    non_opt.add_argument("--hypers_nep", metavar="<float>", type=float, dest="hypers_nep", required=True, nargs="+")
    non_opt.add_argument("--model_path", metavar="<dat>", type=str, dest="model_path", required=True)
    non_opt.add_argument("--gpu_id", metavar="<int>", type=int, dest="gpu_id", required=True)
    non_opt.add_argument("--shape", metavar="<str>", type=str, dest="shape", required=True)
    parser.add_argument("--method", choices=["fd", "fd_split", "adjoint"], default=None)
    parser.add_argument("--activation", choices=["relu", "tanh", "silu"], default="relu")
    parser.add_argument("--nn_width", type=int, default=150)
    parser.add_argument("--nn_hidden", type=int, default=3)
    parser.add_argument("--nve", action="store_true")
    args = parser.parse_args(argv)

    if not os.path.exists("./out/"):
        os.makedirs("./out/")
    gsd_filename = "./out/" + args.output + ".gsd"

    sim = NVT()
    sim.setDevice(args.gpu_id)
    sim.setNNShape(args.nn_width, args.nn_hidden)
    sim.setActivation(args.activation)
    if args.method:
        sim.setForceMethod(args.method)
    sim.setNVE(args.nve)
    sim.initializeSystem(args.init_gsd)
    sim.setNepDescriptors(args.hypers_nep)
    sim.setEvaluator(args.model_path)
    sim.setShape(args.shape)
    sim.setNeighborList()
    sim.setGsdDump(args.dump_period, gsd_filename)
    sim.setkT(args.kT)
    sim.setdt(args.dt)
    sim.run(args.timesteps)
    return sim


if __name__ == "__main__":
    main()
