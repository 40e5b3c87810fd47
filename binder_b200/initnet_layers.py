"""The learned initialiser's layer table (input and output channels of its 11 convolutions in
forward order), shared by the host code that lays out its parameters."""


def layer_table(in_channels=2):
    return [(in_channels, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 128),
            (128, 128), (128, 64), (64, 64), (64, 3)]
