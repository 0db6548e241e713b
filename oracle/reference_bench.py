"""Reference arm of bench.py (test infrastructure): times the reference runtime itself."""
import json


def main(args):
    print(json.dumps({"impl": "reference", "unavailable": "reference CUDA build not wired yet"}))
